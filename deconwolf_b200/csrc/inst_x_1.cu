// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_3_0(const XArgs &, cudaStream_t);
void launch_x_25_0(const XArgs &, cudaStream_t);
void launch_x_63_0(const XArgs &, cudaStream_t);
void launch_x_125_0(const XArgs &, cudaStream_t);
void launch_x_200_0(const XArgs &, cudaStream_t);
void launch_x_315_0(const XArgs &, cudaStream_t);
void launch_x_448_0(const XArgs &, cudaStream_t);
void launch_x_640_0(const XArgs &, cudaStream_t);
void launch_x_864_0(const XArgs &, cudaStream_t);
void launch_x_1152_0(const XArgs &, cudaStream_t);
void launch_x_1568_0(const XArgs &, cudaStream_t);
void launch_x_3_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<3, 1, 1>, 32>(a, st); }
void launch_x_25_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<5, 5, 1>, 16>(a, st); }
void launch_x_63_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 7, 1>, 8>(a, st); }
void launch_x_125_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<5, 5, 5>, 4>(a, st); }
void launch_x_200_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 5, 5>, 2>(a, st); }
void launch_x_200_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<5, 5, 8>, 2>(a, st); else launch_x_200_0(a, st); }
void launch_x_315_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 5, 7>, 2>(a, st); }
void launch_x_315_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 5, 9>, 2>(a, st); else launch_x_315_0(a, st); }
void launch_x_448_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 7, 8>, 2>(a, st); }
void launch_x_448_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 8, 8>, 2>(a, st); else launch_x_448_0(a, st); }
void launch_x_640_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 8, 8>, 2>(a, st); }
void launch_x_640_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 8, 10>, 2>(a, st); else launch_x_640_0(a, st); }
void launch_x_864_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 8, 9>, 2>(a, st); }
void launch_x_864_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 8, 12>, 2>(a, st); else launch_x_864_0(a, st); }
void launch_x_1152_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 8, 12>, 1>(a, st); }
void launch_x_1152_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 12, 12>, 1>(a, st); else launch_x_1152_0(a, st); }
void launch_x_1568_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 8, 14>, 1>(a, st); }
void launch_x_1568_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 14, 14>, 1>(a, st); else launch_x_1568_0(a, st); }
}  // namespace dwcu
