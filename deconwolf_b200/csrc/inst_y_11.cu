// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_15_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 3, 1>>(a, st); }
void launch_y_15_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 5, 1>>(a, st); }
void launch_y_15_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 1, 1>>(a, st); }
void launch_y_48_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 6, 1>>(a, st); }
void launch_y_48_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 8, 1>>(a, st); }
void launch_y_48_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 4, 1>>(a, st); }
void launch_y_98_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 1>>(a, st); }
void launch_y_98_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 14, 1>>(a, st); }
void launch_y_98_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<2, 7, 7>>(a, st); }
void launch_y_168_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 12, 1>>(a, st); }
void launch_y_168_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 14, 1>>(a, st); }
void launch_y_168_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 4, 6>>(a, st); }
void launch_y_256_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 16, 1>>(a, st); }
void launch_y_256_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 4, 8>>(a, st); }
void launch_y_256_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 8, 8>>(a, st); }
void launch_y_392_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 7, 7>>(a, st); }
void launch_y_392_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 7, 8>>(a, st); }
void launch_y_392_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 4, 7>>(a, st); }
void launch_y_560_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 8>>(a, st); }
void launch_y_560_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 7, 10>>(a, st); }
void launch_y_560_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 8, 10>>(a, st); }
void launch_y_756_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 7, 9>>(a, st); }
void launch_y_756_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 7, 12>>(a, st); }
void launch_y_756_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 9, 12>>(a, st); }
void launch_y_1024_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 8>>(a, st); }
void launch_y_1024_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 8, 16>>(a, st); }
void launch_y_1024_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 16, 16>>(a, st); }
void launch_y_1400_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 10, 10>>(a, st); }
void launch_y_1400_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 10, 14>>(a, st); }
void launch_y_1920_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 10, 12>>(a, st); }
void launch_y_1920_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 10, 16>>(a, st); }
void launch_y_1920_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 12, 16>>(a, st); }
void launch_y_2744_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 14, 14>>(a, st); }
}  // namespace dwcu
