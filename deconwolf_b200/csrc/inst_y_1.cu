// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_3_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 1, 1>>(a, st); }
void launch_y_25_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 5, 1>>(a, st); }
void launch_y_63_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 7, 1>>(a, st); }
void launch_y_63_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 9, 1>>(a, st); }
void launch_y_63_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 3, 7>>(a, st); }
void launch_y_125_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 5, 5>>(a, st); }
void launch_y_200_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 5, 5>>(a, st); }
void launch_y_200_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 5, 8>>(a, st); }
void launch_y_200_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 4, 5>>(a, st); }
void launch_y_315_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 5, 7>>(a, st); }
void launch_y_315_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 5, 9>>(a, st); }
void launch_y_315_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 7, 9>>(a, st); }
void launch_y_448_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 7, 8>>(a, st); }
void launch_y_448_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 8, 8>>(a, st); }
void launch_y_448_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 4, 8>>(a, st); }
void launch_y_640_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 8, 8>>(a, st); }
void launch_y_640_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 8, 10>>(a, st); }
void launch_y_640_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 5, 8>>(a, st); }
void launch_y_864_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 8, 9>>(a, st); }
void launch_y_864_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 8, 12>>(a, st); }
void launch_y_864_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 9, 12>>(a, st); }
void launch_y_1152_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 8, 12>>(a, st); }
void launch_y_1152_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 12, 12>>(a, st); }
void launch_y_1152_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 9>>(a, st); }
void launch_y_1568_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 14>>(a, st); }
void launch_y_1568_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 14, 14>>(a, st); }
void launch_y_1568_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 7, 14>>(a, st); }
void launch_y_2160_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 12, 12>>(a, st); }
void launch_y_2160_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 12, 15>>(a, st); }
void launch_y_2160_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 9, 15>>(a, st); }
}  // namespace dwcu
