// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_14_0(const XArgs &, cudaStream_t);
void launch_x_45_0(const XArgs &, cudaStream_t);
void launch_x_96_0(const XArgs &, cudaStream_t);
void launch_x_162_0(const XArgs &, cudaStream_t);
void launch_x_252_0(const XArgs &, cudaStream_t);
void launch_x_384_0(const XArgs &, cudaStream_t);
void launch_x_540_0(const XArgs &, cudaStream_t);
void launch_x_750_0(const XArgs &, cudaStream_t);
void launch_x_1008_0(const XArgs &, cudaStream_t);
void launch_x_1372_0(const XArgs &, cudaStream_t);
void launch_x_1890_0(const XArgs &, cudaStream_t);
void launch_x_14_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 2, 1>, 16>(a, st); }
void launch_x_45_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 5, 1>, 8>(a, st); }
void launch_x_96_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 8, 1>, 8>(a, st); }
void launch_x_96_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 12, 1>, 8>(a, st); else launch_x_96_0(a, st); }
void launch_x_162_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 3, 6>, 2>(a, st); }
void launch_x_162_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<6, 3, 9>, 2>(a, st); else launch_x_162_0(a, st); }
void launch_x_252_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 6, 6>, 2>(a, st); }
void launch_x_252_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<6, 6, 7>, 2>(a, st); else launch_x_252_0(a, st); }
void launch_x_384_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 6, 8>, 2>(a, st); }
void launch_x_384_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<6, 8, 8>, 2>(a, st); else launch_x_384_0(a, st); }
void launch_x_540_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 6, 9>, 2>(a, st); }
void launch_x_540_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 6, 10>, 2>(a, st); else launch_x_540_0(a, st); }
void launch_x_750_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 5, 10>, 2>(a, st); }
void launch_x_750_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 5, 15>, 2>(a, st); else launch_x_750_0(a, st); }
void launch_x_1008_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 8, 9>, 2>(a, st); }
void launch_x_1008_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 8, 14>, 2>(a, st); else launch_x_1008_0(a, st); }
void launch_x_1372_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 14>, 1>(a, st); }
void launch_x_1372_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 14, 14>, 1>(a, st); else launch_x_1372_0(a, st); }
void launch_x_1890_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 9, 14>, 1>(a, st); }
void launch_x_1890_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<14, 9, 15>, 1>(a, st); else launch_x_1890_0(a, st); }
}  // namespace dwcu
