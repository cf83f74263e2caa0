// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_2_0(const XArgs &, cudaStream_t);
void launch_x_24_0(const XArgs &, cudaStream_t);
void launch_x_60_0(const XArgs &, cudaStream_t);
void launch_x_120_0(const XArgs &, cudaStream_t);
void launch_x_196_0(const XArgs &, cudaStream_t);
void launch_x_300_0(const XArgs &, cudaStream_t);
void launch_x_441_0(const XArgs &, cudaStream_t);
void launch_x_630_0(const XArgs &, cudaStream_t);
void launch_x_840_0(const XArgs &, cudaStream_t);
void launch_x_1134_0(const XArgs &, cudaStream_t);
void launch_x_1536_0(const XArgs &, cudaStream_t);
void launch_x_2_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<2, 1, 1>, 32>(a, st); }
void launch_x_24_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<6, 4, 1>, 16>(a, st); }
void launch_x_60_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 6, 1>, 8>(a, st); }
void launch_x_120_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 10, 1>, 8>(a, st); }
void launch_x_120_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 12, 1>, 8>(a, st); else launch_x_120_0(a, st); }
void launch_x_196_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 14, 1>, 8>(a, st); }
void launch_x_300_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 6>, 2>(a, st); }
void launch_x_300_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<6, 5, 10>, 2>(a, st); else launch_x_300_0(a, st); }
void launch_x_441_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 7, 7>, 2>(a, st); }
void launch_x_441_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 7, 9>, 2>(a, st); else launch_x_441_0(a, st); }
void launch_x_630_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 7, 9>, 2>(a, st); }
void launch_x_630_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 7, 10>, 2>(a, st); else launch_x_630_0(a, st); }
void launch_x_840_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 7, 10>, 2>(a, st); }
void launch_x_840_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 7, 12>, 2>(a, st); else launch_x_840_0(a, st); }
void launch_x_1134_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 9, 9>, 2>(a, st); }
void launch_x_1134_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 9, 14>, 2>(a, st); else launch_x_1134_0(a, st); }
void launch_x_1536_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 8, 12>, 1>(a, st); }
void launch_x_1536_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<12, 8, 16>, 1>(a, st); else launch_x_1536_0(a, st); }
}  // namespace dwcu
