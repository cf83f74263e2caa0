// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_20_0(const XArgs &, cudaStream_t);
void launch_x_54_0(const XArgs &, cudaStream_t);
void launch_x_108_0(const XArgs &, cudaStream_t);
void launch_x_189_0(const XArgs &, cudaStream_t);
void launch_x_288_0(const XArgs &, cudaStream_t);
void launch_x_420_0(const XArgs &, cudaStream_t);
void launch_x_588_0(const XArgs &, cudaStream_t);
void launch_x_800_0(const XArgs &, cudaStream_t);
void launch_x_1120_0(const XArgs &, cudaStream_t);
void launch_x_1500_0(const XArgs &, cudaStream_t);
void launch_x_2025_0(const XArgs &, cudaStream_t);
void launch_x_20_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<5, 4, 1>, 16>(a, st); }
void launch_x_54_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 6, 1>, 8>(a, st); }
void launch_x_108_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 9, 1>, 8>(a, st); }
void launch_x_108_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 12, 1>, 8>(a, st); else launch_x_108_0(a, st); }
void launch_x_189_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 3, 7>, 2>(a, st); }
void launch_x_189_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 3, 9>, 2>(a, st); else launch_x_189_0(a, st); }
void launch_x_288_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 6, 6>, 2>(a, st); }
void launch_x_288_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<6, 6, 8>, 2>(a, st); else launch_x_288_0(a, st); }
void launch_x_420_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 6, 7>, 2>(a, st); }
void launch_x_420_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 6, 10>, 2>(a, st); else launch_x_420_0(a, st); }
void launch_x_588_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 7, 7>, 2>(a, st); }
void launch_x_588_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 7, 12>, 2>(a, st); else launch_x_588_0(a, st); }
void launch_x_800_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 8, 10>, 2>(a, st); }
void launch_x_800_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 10, 10>, 2>(a, st); else launch_x_800_0(a, st); }
void launch_x_1120_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 8, 10>, 2>(a, st); }
void launch_x_1120_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 8, 14>, 2>(a, st); else launch_x_1120_0(a, st); }
void launch_x_1500_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 10, 10>, 1>(a, st); }
void launch_x_1500_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 10, 15>, 1>(a, st); else launch_x_1500_0(a, st); }
void launch_x_2025_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 9, 15>, 1>(a, st); }
void launch_x_2025_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 15, 15>, 1>(a, st); else launch_x_2025_0(a, st); }
}  // namespace dwcu
