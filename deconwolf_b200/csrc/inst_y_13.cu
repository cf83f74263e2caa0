// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_18_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 3, 1>>(a, st); }
void launch_y_18_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 6, 1>>(a, st); }
void launch_y_18_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 2, 1>>(a, st); }
void launch_y_50_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 1>>(a, st); }
void launch_y_50_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 10, 1>>(a, st); }
void launch_y_50_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<2, 5, 5>>(a, st); }
void launch_y_105_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 7, 1>>(a, st); }
void launch_y_105_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 15, 1>>(a, st); }
void launch_y_105_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 3, 7>>(a, st); }
void launch_y_180_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 12, 1>>(a, st); }
void launch_y_180_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 15, 1>>(a, st); }
void launch_y_180_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 5, 6>>(a, st); }
void launch_y_280_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 5, 7>>(a, st); }
void launch_y_280_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 5, 8>>(a, st); }
void launch_y_280_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 7, 8>>(a, st); }
void launch_y_405_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 5, 9>>(a, st); }
void launch_y_405_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 9, 9>>(a, st); }
void launch_y_405_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 3, 9>>(a, st); }
void launch_y_576_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 8, 8>>(a, st); }
void launch_y_576_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 8, 9>>(a, st); }
void launch_y_576_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 6, 8>>(a, st); }
void launch_y_784_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 8>>(a, st); }
void launch_y_784_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 7, 14>>(a, st); }
void launch_y_784_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 8, 14>>(a, st); }
void launch_y_1080_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 9, 10>>(a, st); }
void launch_y_1080_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 9, 12>>(a, st); }
void launch_y_1080_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 10, 12>>(a, st); }
void launch_y_1470_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 7, 14>>(a, st); }
void launch_y_1470_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 15>>(a, st); }
void launch_y_1470_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 14, 15>>(a, st); }
void launch_y_2016_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 12, 12>>(a, st); }
void launch_y_2016_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 12, 14>>(a, st); }
void launch_y_2016_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 9, 14>>(a, st); }
void launch_y_2940_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 14, 14>>(a, st); }
void launch_y_2940_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 14, 15>>(a, st); }
}  // namespace dwcu
