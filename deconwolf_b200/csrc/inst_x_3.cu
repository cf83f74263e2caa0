// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_5(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<5, 1, 1>, 16>(a, st); }
void launch_x_28(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 4, 1>, 16>(a, st); }
void launch_x_70(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 7, 1>, 8>(a, st); }
void launch_x_128(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 8, 1>, 4>(a, st); }
void launch_x_216(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<6, 6, 6>, 2>(a, st); }
void launch_x_324(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 6, 6>, 2>(a, st); }
void launch_x_480(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 6, 8>, 2>(a, st); }
void launch_x_672(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 7, 8>, 2>(a, st); }
void launch_x_896(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 8, 8>, 2>(a, st); }
void launch_x_1200(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 10, 10>, 1>(a, st); }
void launch_x_1600(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 10, 10>, 1>(a, st); }
}  // namespace dwcu
