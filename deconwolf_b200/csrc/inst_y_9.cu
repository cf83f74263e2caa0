// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_12_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 3, 1>>(a, st); }
void launch_y_12_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 4, 1>>(a, st); }
void launch_y_12_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 2, 1>>(a, st); }
void launch_y_42_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 6, 1>>(a, st); }
void launch_y_42_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 7, 1>>(a, st); }
void launch_y_42_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 3, 1>>(a, st); }
void launch_y_90_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 9, 1>>(a, st); }
void launch_y_90_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 10, 1>>(a, st); }
void launch_y_90_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 6, 1>>(a, st); }
void launch_y_160_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 10, 1>>(a, st); }
void launch_y_160_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 16, 1>>(a, st); }
void launch_y_160_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 4, 5>>(a, st); }
void launch_y_250_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 5>>(a, st); }
void launch_y_250_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 5, 10>>(a, st); }
void launch_y_378_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 6, 7>>(a, st); }
void launch_y_378_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 6, 9>>(a, st); }
void launch_y_378_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 7, 9>>(a, st); }
void launch_y_525_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 5, 7>>(a, st); }
void launch_y_525_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 5, 15>>(a, st); }
void launch_y_525_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 7, 15>>(a, st); }
void launch_y_735_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 7, 7>>(a, st); }
void launch_y_735_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 7, 15>>(a, st); }
void launch_y_1000_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 10, 10>>(a, st); }
void launch_y_1350_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 9, 10>>(a, st); }
void launch_y_1350_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 9, 15>>(a, st); }
void launch_y_1350_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 10, 15>>(a, st); }
void launch_y_1800_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 10, 12>>(a, st); }
void launch_y_1800_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 10, 15>>(a, st); }
void launch_y_1800_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 12, 15>>(a, st); }
void launch_y_2688_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 12, 14>>(a, st); }
void launch_y_2688_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 12, 16>>(a, st); }
void launch_y_2688_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 14, 16>>(a, st); }
}  // namespace dwcu
