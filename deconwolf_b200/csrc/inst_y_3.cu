// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_5_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 1, 1>>(a, st); }
void launch_y_28_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 4, 1>>(a, st); }
void launch_y_28_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 7, 1>>(a, st); }
void launch_y_28_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 2, 1>>(a, st); }
void launch_y_70_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 1>>(a, st); }
void launch_y_70_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 10, 1>>(a, st); }
void launch_y_70_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 5, 1>>(a, st); }
void launch_y_128_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 1>>(a, st); }
void launch_y_128_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 16, 1>>(a, st); }
void launch_y_128_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 4, 8>>(a, st); }
void launch_y_216_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 6, 6>>(a, st); }
void launch_y_216_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 4, 6>>(a, st); }
void launch_y_216_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 6, 9>>(a, st); }
void launch_y_324_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 6, 6>>(a, st); }
void launch_y_324_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 6, 9>>(a, st); }
void launch_y_324_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 9, 9>>(a, st); }
void launch_y_480_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 6, 8>>(a, st); }
void launch_y_480_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 6, 10>>(a, st); }
void launch_y_480_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 8, 10>>(a, st); }
void launch_y_672_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 7, 8>>(a, st); }
void launch_y_672_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 7, 12>>(a, st); }
void launch_y_672_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 8, 12>>(a, st); }
void launch_y_896_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 8>>(a, st); }
void launch_y_896_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 8, 14>>(a, st); }
void launch_y_896_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 7, 8>>(a, st); }
void launch_y_1200_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 10, 10>>(a, st); }
void launch_y_1200_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 10, 12>>(a, st); }
void launch_y_1200_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 8, 10>>(a, st); }
void launch_y_1600_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 10, 10>>(a, st); }
void launch_y_1600_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 10, 16>>(a, st); }
void launch_y_2250_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 10, 15>>(a, st); }
void launch_y_2250_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 15, 15>>(a, st); }
}  // namespace dwcu
