// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_12_0(const XArgs &, cudaStream_t);
void launch_x_42_0(const XArgs &, cudaStream_t);
void launch_x_90_0(const XArgs &, cudaStream_t);
void launch_x_160_0(const XArgs &, cudaStream_t);
void launch_x_250_0(const XArgs &, cudaStream_t);
void launch_x_378_0(const XArgs &, cudaStream_t);
void launch_x_525_0(const XArgs &, cudaStream_t);
void launch_x_735_0(const XArgs &, cudaStream_t);
void launch_x_1000_0(const XArgs &, cudaStream_t);
void launch_x_1350_0(const XArgs &, cudaStream_t);
void launch_x_1800_0(const XArgs &, cudaStream_t);
void launch_x_12_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<4, 3, 1>, 16>(a, st); }
void launch_x_42_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 6, 1>, 16>(a, st); }
void launch_x_90_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 9, 1>, 8>(a, st); }
void launch_x_160_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 10, 1>, 4>(a, st); }
void launch_x_160_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 16, 1>, 4>(a, st); else launch_x_160_0(a, st); }
void launch_x_250_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 5>, 2>(a, st); }
void launch_x_250_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<5, 5, 10>, 2>(a, st); else launch_x_250_0(a, st); }
void launch_x_378_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 6, 7>, 2>(a, st); }
void launch_x_378_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 6, 9>, 2>(a, st); else launch_x_378_0(a, st); }
void launch_x_525_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 5, 7>, 2>(a, st); }
void launch_x_525_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 5, 15>, 2>(a, st); else launch_x_525_0(a, st); }
void launch_x_735_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 7, 7>, 2>(a, st); }
void launch_x_735_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 7, 15>, 2>(a, st); else launch_x_735_0(a, st); }
void launch_x_1000_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 10, 10>, 2>(a, st); }
void launch_x_1350_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 9, 10>, 1>(a, st); }
void launch_x_1350_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 9, 15>, 1>(a, st); else launch_x_1350_0(a, st); }
void launch_x_1800_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 10, 12>, 1>(a, st); }
void launch_x_1800_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<12, 10, 15>, 1>(a, st); else launch_x_1800_0(a, st); }
}  // namespace dwcu
