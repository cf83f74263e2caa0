// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_4_0(const XArgs &, cudaStream_t);
void launch_x_27_0(const XArgs &, cudaStream_t);
void launch_x_64_0(const XArgs &, cudaStream_t);
void launch_x_126_0(const XArgs &, cudaStream_t);
void launch_x_210_0(const XArgs &, cudaStream_t);
void launch_x_320_0(const XArgs &, cudaStream_t);
void launch_x_450_0(const XArgs &, cudaStream_t);
void launch_x_648_0(const XArgs &, cudaStream_t);
void launch_x_882_0(const XArgs &, cudaStream_t);
void launch_x_1176_0(const XArgs &, cudaStream_t);
void launch_x_1575_0(const XArgs &, cudaStream_t);
void launch_x_4_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<2, 2, 1>, 32>(a, st); }
void launch_x_27_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 3, 1>, 8>(a, st); }
void launch_x_64_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 8, 1>, 8>(a, st); }
void launch_x_126_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 9, 1>, 8>(a, st); }
void launch_x_126_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 14, 1>, 8>(a, st); else launch_x_126_0(a, st); }
void launch_x_210_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 14, 1>, 8>(a, st); }
void launch_x_210_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<14, 15, 1>, 8>(a, st); else launch_x_210_0(a, st); }
void launch_x_320_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 5, 8>, 2>(a, st); }
void launch_x_320_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<5, 8, 8>, 2>(a, st); else launch_x_320_0(a, st); }
void launch_x_450_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 9>, 2>(a, st); }
void launch_x_450_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 5, 10>, 2>(a, st); else launch_x_450_0(a, st); }
void launch_x_648_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 8, 9>, 2>(a, st); }
void launch_x_648_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 9, 9>, 2>(a, st); else launch_x_648_0(a, st); }
void launch_x_882_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 9>, 2>(a, st); }
void launch_x_882_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 7, 14>, 2>(a, st); else launch_x_882_0(a, st); }
void launch_x_1176_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 12>, 1>(a, st); }
void launch_x_1176_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<12, 7, 14>, 1>(a, st); else launch_x_1176_0(a, st); }
void launch_x_1575_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 7, 15>, 1>(a, st); }
void launch_x_1575_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 15, 15>, 1>(a, st); else launch_x_1575_0(a, st); }
}  // namespace dwcu
