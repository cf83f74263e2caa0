// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_14_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 2, 1>>(a, st); }
void launch_y_14_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<2, 7, 1>>(a, st); }
void launch_y_14_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 1, 1>>(a, st); }
void launch_y_45_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 5, 1>>(a, st); }
void launch_y_45_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 9, 1>>(a, st); }
void launch_y_45_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 3, 1>>(a, st); }
void launch_y_96_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 8, 1>>(a, st); }
void launch_y_96_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 12, 1>>(a, st); }
void launch_y_96_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 6, 1>>(a, st); }
void launch_y_162_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 3, 6>>(a, st); }
void launch_y_162_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 3, 9>>(a, st); }
void launch_y_162_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 6, 9>>(a, st); }
void launch_y_252_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 6, 6>>(a, st); }
void launch_y_252_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 6, 7>>(a, st); }
void launch_y_252_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 4, 7>>(a, st); }
void launch_y_384_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 6, 8>>(a, st); }
void launch_y_384_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 8, 8>>(a, st); }
void launch_y_384_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 4, 8>>(a, st); }
void launch_y_540_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 6, 9>>(a, st); }
void launch_y_540_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 6, 10>>(a, st); }
void launch_y_540_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 9, 10>>(a, st); }
void launch_y_750_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 5, 10>>(a, st); }
void launch_y_750_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 15>>(a, st); }
void launch_y_750_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 10, 15>>(a, st); }
void launch_y_1008_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 9>>(a, st); }
void launch_y_1008_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 8, 14>>(a, st); }
void launch_y_1008_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 9, 14>>(a, st); }
void launch_y_1372_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 14>>(a, st); }
void launch_y_1372_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 14, 14>>(a, st); }
void launch_y_1890_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 9, 14>>(a, st); }
void launch_y_1890_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 9, 15>>(a, st); }
void launch_y_1890_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 14, 15>>(a, st); }
void launch_y_2700_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 12, 15>>(a, st); }
void launch_y_2700_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 15, 15>>(a, st); }
}  // namespace dwcu
