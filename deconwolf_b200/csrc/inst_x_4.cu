// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_6_0(const XArgs &, cudaStream_t);
void launch_x_30_0(const XArgs &, cudaStream_t);
void launch_x_72_0(const XArgs &, cudaStream_t);
void launch_x_135_0(const XArgs &, cudaStream_t);
void launch_x_224_0(const XArgs &, cudaStream_t);
void launch_x_336_0(const XArgs &, cudaStream_t);
void launch_x_486_0(const XArgs &, cudaStream_t);
void launch_x_675_0(const XArgs &, cudaStream_t);
void launch_x_900_0(const XArgs &, cudaStream_t);
void launch_x_1215_0(const XArgs &, cudaStream_t);
void launch_x_1620_0(const XArgs &, cudaStream_t);
void launch_x_6_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<3, 2, 1>, 32>(a, st); }
void launch_x_30_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<6, 5, 1>, 16>(a, st); }
void launch_x_72_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 8, 1>, 8>(a, st); }
void launch_x_135_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 9, 1>, 8>(a, st); }
void launch_x_135_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 15, 1>, 8>(a, st); else launch_x_135_0(a, st); }
void launch_x_224_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 14, 1>, 4>(a, st); }
void launch_x_224_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<14, 16, 1>, 4>(a, st); else launch_x_224_0(a, st); }
void launch_x_336_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 6, 7>, 2>(a, st); }
void launch_x_336_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 6, 8>, 2>(a, st); else launch_x_336_0(a, st); }
void launch_x_486_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 6, 9>, 2>(a, st); }
void launch_x_486_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<6, 9, 9>, 2>(a, st); else launch_x_486_0(a, st); }
void launch_x_675_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 5, 9>, 2>(a, st); }
void launch_x_675_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 5, 15>, 2>(a, st); else launch_x_675_0(a, st); }
void launch_x_900_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 9, 10>, 2>(a, st); }
void launch_x_900_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 10, 10>, 2>(a, st); else launch_x_900_0(a, st); }
void launch_x_1215_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 9, 9>, 1>(a, st); }
void launch_x_1215_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 9, 15>, 1>(a, st); else launch_x_1215_0(a, st); }
void launch_x_1620_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 9, 12>, 1>(a, st); }
void launch_x_1620_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<12, 9, 15>, 1>(a, st); else launch_x_1620_0(a, st); }
}  // namespace dwcu
