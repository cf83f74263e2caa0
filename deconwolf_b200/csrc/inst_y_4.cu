// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_6_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 2, 1>>(a, st); }
void launch_y_6_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<2, 3, 1>>(a, st); }
void launch_y_6_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 1, 1>>(a, st); }
void launch_y_30_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 5, 1>>(a, st); }
void launch_y_30_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 6, 1>>(a, st); }
void launch_y_30_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 3, 1>>(a, st); }
void launch_y_72_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 8, 1>>(a, st); }
void launch_y_72_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 9, 1>>(a, st); }
void launch_y_72_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 6, 1>>(a, st); }
void launch_y_135_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 9, 1>>(a, st); }
void launch_y_135_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 15, 1>>(a, st); }
void launch_y_135_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 3, 9>>(a, st); }
void launch_y_224_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 14, 1>>(a, st); }
void launch_y_224_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 16, 1>>(a, st); }
void launch_y_224_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 4, 7>>(a, st); }
void launch_y_336_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 6, 7>>(a, st); }
void launch_y_336_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 6, 8>>(a, st); }
void launch_y_336_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 7, 8>>(a, st); }
void launch_y_486_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 6, 9>>(a, st); }
void launch_y_486_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 9, 9>>(a, st); }
void launch_y_675_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 5, 9>>(a, st); }
void launch_y_675_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 5, 15>>(a, st); }
void launch_y_675_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 9, 15>>(a, st); }
void launch_y_900_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 9, 10>>(a, st); }
void launch_y_900_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 10, 10>>(a, st); }
void launch_y_900_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 6, 10>>(a, st); }
void launch_y_1215_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 9, 9>>(a, st); }
void launch_y_1215_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 9, 15>>(a, st); }
void launch_y_1620_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 9, 12>>(a, st); }
void launch_y_1620_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 9, 15>>(a, st); }
void launch_y_1620_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 12, 15>>(a, st); }
void launch_y_2304_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 12, 12>>(a, st); }
void launch_y_2304_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 12, 16>>(a, st); }
void launch_y_2304_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 16, 16>>(a, st); }
}  // namespace dwcu
