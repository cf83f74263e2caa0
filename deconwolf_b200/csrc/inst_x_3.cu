// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_5_0(const XArgs &, cudaStream_t);
void launch_x_28_0(const XArgs &, cudaStream_t);
void launch_x_70_0(const XArgs &, cudaStream_t);
void launch_x_128_0(const XArgs &, cudaStream_t);
void launch_x_216_0(const XArgs &, cudaStream_t);
void launch_x_324_0(const XArgs &, cudaStream_t);
void launch_x_480_0(const XArgs &, cudaStream_t);
void launch_x_672_0(const XArgs &, cudaStream_t);
void launch_x_896_0(const XArgs &, cudaStream_t);
void launch_x_1200_0(const XArgs &, cudaStream_t);
void launch_x_1600_0(const XArgs &, cudaStream_t);
void launch_x_5_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<5, 1, 1>, 16>(a, st); }
void launch_x_28_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 4, 1>, 16>(a, st); }
void launch_x_70_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 7, 1>, 8>(a, st); }
void launch_x_128_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 8, 1>, 4>(a, st); }
void launch_x_128_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 16, 1>, 4>(a, st); else launch_x_128_0(a, st); }
void launch_x_216_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<6, 6, 6>, 2>(a, st); }
void launch_x_216_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<9, 4, 6>, 2>(a, st); else launch_x_216_0(a, st); }
void launch_x_324_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 6, 6>, 2>(a, st); }
void launch_x_324_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<6, 6, 9>, 2>(a, st); else launch_x_324_0(a, st); }
void launch_x_480_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 6, 8>, 2>(a, st); }
void launch_x_480_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 6, 10>, 2>(a, st); else launch_x_480_0(a, st); }
void launch_x_672_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 7, 8>, 2>(a, st); }
void launch_x_672_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 7, 12>, 2>(a, st); else launch_x_672_0(a, st); }
void launch_x_896_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 8, 8>, 2>(a, st); }
void launch_x_896_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<8, 8, 14>, 2>(a, st); else launch_x_896_0(a, st); }
void launch_x_1200_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 10, 10>, 1>(a, st); }
void launch_x_1200_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 10, 12>, 1>(a, st); else launch_x_1200_0(a, st); }
void launch_x_1600_0(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 10, 10>, 1>(a, st); }
void launch_x_1600_1(const XArgs &a, cudaStream_t st) { if (x_iteration_op(a.op)) launch_x_iter_t<Rad<10, 10, 16>, 1>(a, st); else launch_x_1600_0(a, st); }
}  // namespace dwcu
