// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_21_0(const XArgs &, cudaStream_t);
void launch_x_56_0(const XArgs &, cudaStream_t);
void launch_x_112_0(const XArgs &, cudaStream_t);
void launch_x_192_0(const XArgs &, cudaStream_t);
void launch_x_294_0(const XArgs &, cudaStream_t);
void launch_x_432_0(const XArgs &, cudaStream_t);
void launch_x_600_0(const XArgs &, cudaStream_t);
void launch_x_810_0(const XArgs &, cudaStream_t);
void launch_x_1125_0(const XArgs &, cudaStream_t);
void launch_x_1512_0(const XArgs &, cudaStream_t);
void launch_x_2048_0(const XArgs &, cudaStream_t);
void launch_x_21_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 3, 1>, 16>(a, st); }
void launch_x_56_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 7, 1>, 8>(a, st); }
void launch_x_112_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 8, 1>, 8>(a, st); }
void launch_x_112_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 14, 1>, 8>(a, st); else launch_x_112_0(a, st); }
void launch_x_192_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 12, 1>, 4>(a, st); }
void launch_x_192_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<12, 16, 1>, 4>(a, st); else launch_x_192_0(a, st); }
void launch_x_294_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 6, 7>, 2>(a, st); }
void launch_x_294_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<6, 7, 7>, 2>(a, st); else launch_x_294_0(a, st); }
void launch_x_432_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 6, 8>, 2>(a, st); }
void launch_x_432_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 6, 9>, 2>(a, st); else launch_x_432_0(a, st); }
void launch_x_600_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 6, 10>, 2>(a, st); }
void launch_x_600_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<6, 10, 10>, 2>(a, st); else launch_x_600_0(a, st); }
void launch_x_810_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 9, 9>, 2>(a, st); }
void launch_x_810_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 9, 10>, 2>(a, st); else launch_x_810_0(a, st); }
void launch_x_1125_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 5, 15>, 1>(a, st); }
void launch_x_1125_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<5, 15, 15>, 1>(a, st); else launch_x_1125_0(a, st); }
void launch_x_1512_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 9, 12>, 1>(a, st); }
void launch_x_1512_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<12, 9, 14>, 1>(a, st); else launch_x_1512_0(a, st); }
void launch_x_2048_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 8, 16>, 1>(a, st); }
void launch_x_2048_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 16, 16>, 1>(a, st); else launch_x_2048_0(a, st); }
}  // namespace dwcu
