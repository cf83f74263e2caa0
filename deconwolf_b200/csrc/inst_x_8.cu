// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_10_0(const XArgs &, cudaStream_t);
void launch_x_40_0(const XArgs &, cudaStream_t);
void launch_x_84_0(const XArgs &, cudaStream_t);
void launch_x_150_0(const XArgs &, cudaStream_t);
void launch_x_245_0(const XArgs &, cudaStream_t);
void launch_x_375_0(const XArgs &, cudaStream_t);
void launch_x_512_0(const XArgs &, cudaStream_t);
void launch_x_729_0(const XArgs &, cudaStream_t);
void launch_x_980_0(const XArgs &, cudaStream_t);
void launch_x_1344_0(const XArgs &, cudaStream_t);
void launch_x_1792_0(const XArgs &, cudaStream_t);
void launch_x_10_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<5, 2, 1>, 16>(a, st); }
void launch_x_40_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 5, 1>, 8>(a, st); }
void launch_x_84_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 7, 1>, 8>(a, st); }
void launch_x_150_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 10, 1>, 8>(a, st); }
void launch_x_150_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 15, 1>, 8>(a, st); else launch_x_150_0(a, st); }
void launch_x_245_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 5, 7>, 2>(a, st); }
void launch_x_245_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<5, 7, 7>, 2>(a, st); else launch_x_245_0(a, st); }
void launch_x_375_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 5, 5>, 2>(a, st); }
void launch_x_375_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<5, 5, 15>, 2>(a, st); else launch_x_375_0(a, st); }
void launch_x_512_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 8, 8>, 2>(a, st); }
void launch_x_512_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<16, 4, 8>, 2>(a, st); else launch_x_512_0(a, st); }
void launch_x_729_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 9, 9>, 2>(a, st); }
void launch_x_980_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 10>, 2>(a, st); }
void launch_x_980_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 7, 14>, 2>(a, st); else launch_x_980_0(a, st); }
void launch_x_1344_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 8, 12>, 1>(a, st); }
void launch_x_1344_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<12, 8, 14>, 1>(a, st); else launch_x_1344_0(a, st); }
void launch_x_1792_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 8, 14>, 1>(a, st); }
void launch_x_1792_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<14, 8, 16>, 1>(a, st); else launch_x_1792_0(a, st); }
}  // namespace dwcu
