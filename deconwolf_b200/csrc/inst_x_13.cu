// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_18_0(const XArgs &, cudaStream_t);
void launch_x_50_0(const XArgs &, cudaStream_t);
void launch_x_105_0(const XArgs &, cudaStream_t);
void launch_x_180_0(const XArgs &, cudaStream_t);
void launch_x_280_0(const XArgs &, cudaStream_t);
void launch_x_405_0(const XArgs &, cudaStream_t);
void launch_x_576_0(const XArgs &, cudaStream_t);
void launch_x_784_0(const XArgs &, cudaStream_t);
void launch_x_1080_0(const XArgs &, cudaStream_t);
void launch_x_1470_0(const XArgs &, cudaStream_t);
void launch_x_2016_0(const XArgs &, cudaStream_t);
void launch_x_18_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<6, 3, 1>, 16>(a, st); }
void launch_x_50_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 1>, 8>(a, st); }
void launch_x_105_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 7, 1>, 8>(a, st); }
void launch_x_105_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 15, 1>, 8>(a, st); else launch_x_105_0(a, st); }
void launch_x_180_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 12, 1>, 8>(a, st); }
void launch_x_180_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<12, 15, 1>, 8>(a, st); else launch_x_180_0(a, st); }
void launch_x_280_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 5, 7>, 2>(a, st); }
void launch_x_280_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 5, 8>, 2>(a, st); else launch_x_280_0(a, st); }
void launch_x_405_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 5, 9>, 2>(a, st); }
void launch_x_405_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<5, 9, 9>, 2>(a, st); else launch_x_405_0(a, st); }
void launch_x_576_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 8, 8>, 2>(a, st); }
void launch_x_576_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 8, 9>, 2>(a, st); else launch_x_576_0(a, st); }
void launch_x_784_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 8>, 2>(a, st); }
void launch_x_784_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 7, 14>, 2>(a, st); else launch_x_784_0(a, st); }
void launch_x_1080_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 9, 10>, 2>(a, st); }
void launch_x_1080_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 9, 12>, 2>(a, st); else launch_x_1080_0(a, st); }
void launch_x_1470_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 7, 14>, 1>(a, st); }
void launch_x_1470_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<14, 7, 15>, 1>(a, st); else launch_x_1470_0(a, st); }
void launch_x_2016_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 12, 12>, 1>(a, st); }
void launch_x_2016_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<12, 12, 14>, 1>(a, st); else launch_x_2016_0(a, st); }
}  // namespace dwcu
