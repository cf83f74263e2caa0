// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_16_0(const XArgs &, cudaStream_t);
void launch_x_49_0(const XArgs &, cudaStream_t);
void launch_x_100_0(const XArgs &, cudaStream_t);
void launch_x_175_0(const XArgs &, cudaStream_t);
void launch_x_270_0(const XArgs &, cudaStream_t);
void launch_x_400_0(const XArgs &, cudaStream_t);
void launch_x_567_0(const XArgs &, cudaStream_t);
void launch_x_768_0(const XArgs &, cudaStream_t);
void launch_x_1050_0(const XArgs &, cudaStream_t);
void launch_x_1440_0(const XArgs &, cudaStream_t);
void launch_x_1960_0(const XArgs &, cudaStream_t);
void launch_x_16_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<4, 4, 1>, 16>(a, st); }
void launch_x_49_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 7, 1>, 16>(a, st); }
void launch_x_100_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 10, 1>, 8>(a, st); }
void launch_x_175_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 5, 5>, 2>(a, st); }
void launch_x_175_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<5, 5, 7>, 2>(a, st); else launch_x_175_0(a, st); }
void launch_x_270_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 5, 6>, 2>(a, st); }
void launch_x_270_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<6, 5, 9>, 2>(a, st); else launch_x_270_0(a, st); }
void launch_x_400_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 8>, 2>(a, st); }
void launch_x_400_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 5, 10>, 2>(a, st); else launch_x_400_0(a, st); }
void launch_x_567_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 7, 9>, 2>(a, st); }
void launch_x_567_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 9, 9>, 2>(a, st); else launch_x_567_0(a, st); }
void launch_x_768_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 8, 8>, 2>(a, st); }
void launch_x_768_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 8, 12>, 2>(a, st); else launch_x_768_0(a, st); }
void launch_x_1050_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 7, 10>, 2>(a, st); }
void launch_x_1050_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 7, 15>, 2>(a, st); else launch_x_1050_0(a, st); }
void launch_x_1440_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 10, 12>, 1>(a, st); }
void launch_x_1440_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 12, 12>, 1>(a, st); else launch_x_1440_0(a, st); }
void launch_x_1960_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 10, 14>, 1>(a, st); }
void launch_x_1960_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 14, 14>, 1>(a, st); else launch_x_1960_0(a, st); }
}  // namespace dwcu
