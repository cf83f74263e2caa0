// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_5(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 1, 1>>(a, st); }
void launch_y_28(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 4, 1>>(a, st); }
void launch_y_70(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 1>>(a, st); }
void launch_y_128(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 1>>(a, st); }
void launch_y_216(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 6, 6>>(a, st); }
void launch_y_324(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 6, 6>>(a, st); }
void launch_y_480(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 6, 8>>(a, st); }
void launch_y_672(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 7, 8>>(a, st); }
void launch_y_896(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 8>>(a, st); }
void launch_y_1200(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 10, 10>>(a, st); }
void launch_y_1600(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 10, 10>>(a, st); }
void launch_y_2250(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 10, 15>>(a, st); }
}  // namespace dwcu
