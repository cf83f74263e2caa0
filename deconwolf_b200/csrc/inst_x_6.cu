// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_8_0(const XArgs &, cudaStream_t);
void launch_x_35_0(const XArgs &, cudaStream_t);
void launch_x_80_0(const XArgs &, cudaStream_t);
void launch_x_144_0(const XArgs &, cudaStream_t);
void launch_x_240_0(const XArgs &, cudaStream_t);
void launch_x_350_0(const XArgs &, cudaStream_t);
void launch_x_500_0(const XArgs &, cudaStream_t);
void launch_x_700_0(const XArgs &, cudaStream_t);
void launch_x_960_0(const XArgs &, cudaStream_t);
void launch_x_1280_0(const XArgs &, cudaStream_t);
void launch_x_1728_0(const XArgs &, cudaStream_t);
void launch_x_8_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<4, 2, 1>, 16>(a, st); }
void launch_x_35_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 5, 1>, 16>(a, st); }
void launch_x_80_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 8, 1>, 8>(a, st); }
void launch_x_144_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 12, 1>, 8>(a, st); }
void launch_x_240_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 15, 1>, 4>(a, st); }
void launch_x_240_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<15, 16, 1>, 4>(a, st); else launch_x_240_0(a, st); }
void launch_x_350_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 7>, 2>(a, st); }
void launch_x_350_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 5, 10>, 2>(a, st); else launch_x_350_0(a, st); }
void launch_x_500_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 10>, 2>(a, st); }
void launch_x_500_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<5, 10, 10>, 2>(a, st); else launch_x_500_0(a, st); }
void launch_x_700_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 7, 10>, 2>(a, st); }
void launch_x_700_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<7, 10, 10>, 2>(a, st); else launch_x_700_0(a, st); }
void launch_x_960_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 8, 10>, 2>(a, st); }
void launch_x_960_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 8, 12>, 2>(a, st); else launch_x_960_0(a, st); }
void launch_x_1280_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 8, 10>, 1>(a, st); }
void launch_x_1280_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 8, 16>, 1>(a, st); else launch_x_1280_0(a, st); }
void launch_x_1728_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 12, 12>, 1>(a, st); }
void launch_x_1728_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<16, 9, 12>, 1>(a, st); else launch_x_1728_0(a, st); }
}  // namespace dwcu
