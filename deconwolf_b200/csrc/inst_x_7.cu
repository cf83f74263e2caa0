// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_9_0(const XArgs &, cudaStream_t);
void launch_x_36_0(const XArgs &, cudaStream_t);
void launch_x_81_0(const XArgs &, cudaStream_t);
void launch_x_147_0(const XArgs &, cudaStream_t);
void launch_x_243_0(const XArgs &, cudaStream_t);
void launch_x_360_0(const XArgs &, cudaStream_t);
void launch_x_504_0(const XArgs &, cudaStream_t);
void launch_x_720_0(const XArgs &, cudaStream_t);
void launch_x_972_0(const XArgs &, cudaStream_t);
void launch_x_1296_0(const XArgs &, cudaStream_t);
void launch_x_1764_0(const XArgs &, cudaStream_t);
void launch_x_9_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<3, 3, 1>, 32>(a, st); }
void launch_x_36_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<6, 6, 1>, 16>(a, st); }
void launch_x_81_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 9, 1>, 8>(a, st); }
void launch_x_147_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 3, 7>, 2>(a, st); }
void launch_x_147_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<3, 7, 7>, 2>(a, st); else launch_x_147_0(a, st); }
void launch_x_243_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 3, 9>, 2>(a, st); }
void launch_x_243_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<3, 9, 9>, 2>(a, st); else launch_x_243_0(a, st); }
void launch_x_360_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 6, 6>, 2>(a, st); }
void launch_x_360_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<6, 6, 10>, 2>(a, st); else launch_x_360_0(a, st); }
void launch_x_504_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 7, 8>, 2>(a, st); }
void launch_x_504_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 7, 9>, 2>(a, st); else launch_x_504_0(a, st); }
void launch_x_720_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 8, 9>, 2>(a, st); }
void launch_x_720_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 8, 10>, 2>(a, st); else launch_x_720_0(a, st); }
void launch_x_972_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 9, 9>, 2>(a, st); }
void launch_x_972_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 9, 12>, 2>(a, st); else launch_x_972_0(a, st); }
void launch_x_1296_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 9, 12>, 1>(a, st); }
void launch_x_1296_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 12, 12>, 1>(a, st); else launch_x_1296_0(a, st); }
void launch_x_1764_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 9, 14>, 1>(a, st); }
void launch_x_1764_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 14, 14>, 1>(a, st); else launch_x_1764_0(a, st); }
}  // namespace dwcu
