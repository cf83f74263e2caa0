// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_16_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 4, 1>>(a, st); }
void launch_y_16_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 2, 1>>(a, st); }
void launch_y_16_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<2, 8, 1>>(a, st); }
void launch_y_49_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 7, 1>>(a, st); }
void launch_y_100_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 10, 1>>(a, st); }
void launch_y_100_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 4, 5>>(a, st); }
void launch_y_100_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 5, 5>>(a, st); }
void launch_y_175_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 5, 5>>(a, st); }
void launch_y_175_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 5, 7>>(a, st); }
void launch_y_270_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 5, 6>>(a, st); }
void launch_y_270_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 5, 9>>(a, st); }
void launch_y_270_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 6, 9>>(a, st); }
void launch_y_400_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 8>>(a, st); }
void launch_y_400_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 5, 10>>(a, st); }
void launch_y_400_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 8, 10>>(a, st); }
void launch_y_567_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 7, 9>>(a, st); }
void launch_y_567_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 9, 9>>(a, st); }
void launch_y_768_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 8, 8>>(a, st); }
void launch_y_768_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 8, 12>>(a, st); }
void launch_y_768_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 6, 8>>(a, st); }
void launch_y_1050_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 7, 10>>(a, st); }
void launch_y_1050_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 15>>(a, st); }
void launch_y_1050_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 10, 15>>(a, st); }
void launch_y_1440_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 10, 12>>(a, st); }
void launch_y_1440_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 12, 12>>(a, st); }
void launch_y_1440_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 9, 10>>(a, st); }
void launch_y_1960_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 10, 14>>(a, st); }
void launch_y_1960_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 14, 14>>(a, st); }
void launch_y_2880_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 12, 15>>(a, st); }
void launch_y_2880_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 12, 16>>(a, st); }
void launch_y_2880_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 15, 16>>(a, st); }
}  // namespace dwcu
