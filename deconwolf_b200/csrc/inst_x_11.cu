// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_15_0(const XArgs &, cudaStream_t);
void launch_x_48_0(const XArgs &, cudaStream_t);
void launch_x_98_0(const XArgs &, cudaStream_t);
void launch_x_168_0(const XArgs &, cudaStream_t);
void launch_x_256_0(const XArgs &, cudaStream_t);
void launch_x_392_0(const XArgs &, cudaStream_t);
void launch_x_560_0(const XArgs &, cudaStream_t);
void launch_x_756_0(const XArgs &, cudaStream_t);
void launch_x_1024_0(const XArgs &, cudaStream_t);
void launch_x_1400_0(const XArgs &, cudaStream_t);
void launch_x_1920_0(const XArgs &, cudaStream_t);
void launch_x_15_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<5, 3, 1>, 16>(a, st); }
void launch_x_48_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 6, 1>, 8>(a, st); }
void launch_x_98_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 1>, 8>(a, st); }
void launch_x_98_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 14, 1>, 8>(a, st); else launch_x_98_0(a, st); }
void launch_x_168_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 12, 1>, 8>(a, st); }
void launch_x_168_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<12, 14, 1>, 8>(a, st); else launch_x_168_0(a, st); }
void launch_x_256_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 16, 1>, 4>(a, st); }
void launch_x_392_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 7, 7>, 2>(a, st); }
void launch_x_392_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 7, 8>, 2>(a, st); else launch_x_392_0(a, st); }
void launch_x_560_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 7, 8>, 2>(a, st); }
void launch_x_560_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 7, 10>, 2>(a, st); else launch_x_560_0(a, st); }
void launch_x_756_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 7, 9>, 2>(a, st); }
void launch_x_756_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 7, 12>, 2>(a, st); else launch_x_756_0(a, st); }
void launch_x_1024_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 8, 8>, 2>(a, st); }
void launch_x_1024_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 8, 16>, 2>(a, st); else launch_x_1024_0(a, st); }
void launch_x_1400_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 10, 10>, 1>(a, st); }
void launch_x_1400_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 10, 14>, 1>(a, st); else launch_x_1400_0(a, st); }
void launch_x_1920_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 10, 12>, 1>(a, st); }
void launch_x_1920_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<12, 10, 16>, 1>(a, st); else launch_x_1920_0(a, st); }
}  // namespace dwcu
