// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_7_0(const XArgs &, cudaStream_t);
void launch_x_32_0(const XArgs &, cudaStream_t);
void launch_x_75_0(const XArgs &, cudaStream_t);
void launch_x_140_0(const XArgs &, cudaStream_t);
void launch_x_225_0(const XArgs &, cudaStream_t);
void launch_x_343_0(const XArgs &, cudaStream_t);
void launch_x_490_0(const XArgs &, cudaStream_t);
void launch_x_686_0(const XArgs &, cudaStream_t);
void launch_x_945_0(const XArgs &, cudaStream_t);
void launch_x_1260_0(const XArgs &, cudaStream_t);
void launch_x_1680_0(const XArgs &, cudaStream_t);
void launch_x_7_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 1, 1>, 16>(a, st); }
void launch_x_32_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 4, 1>, 8>(a, st); }
void launch_x_75_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 5, 1>, 8>(a, st); }
void launch_x_140_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 10, 1>, 8>(a, st); }
void launch_x_140_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 14, 1>, 8>(a, st); else launch_x_140_0(a, st); }
void launch_x_225_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 15, 1>, 8>(a, st); }
void launch_x_343_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 7, 7>, 2>(a, st); }
void launch_x_490_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 7, 7>, 2>(a, st); }
void launch_x_490_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 7, 10>, 2>(a, st); else launch_x_490_0(a, st); }
void launch_x_686_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 7>, 2>(a, st); }
void launch_x_686_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 7, 14>, 2>(a, st); else launch_x_686_0(a, st); }
void launch_x_945_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 7, 9>, 2>(a, st); }
void launch_x_945_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 7, 15>, 2>(a, st); else launch_x_945_0(a, st); }
void launch_x_1260_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 9, 10>, 1>(a, st); }
void launch_x_1260_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 9, 14>, 1>(a, st); else launch_x_1260_0(a, st); }
void launch_x_1680_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 10, 12>, 1>(a, st); }
void launch_x_1680_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<12, 10, 14>, 1>(a, st); else launch_x_1680_0(a, st); }
}  // namespace dwcu
