// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_4_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<2, 2, 1>>(a, st); }
void launch_y_4_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 1, 1>>(a, st); }
void launch_y_27_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 3, 1>>(a, st); }
void launch_y_27_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 9, 1>>(a, st); }
void launch_y_64_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 8, 1>>(a, st); }
void launch_y_64_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 4, 1>>(a, st); }
void launch_y_64_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 16, 1>>(a, st); }
void launch_y_126_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 9, 1>>(a, st); }
void launch_y_126_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 14, 1>>(a, st); }
void launch_y_126_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 3, 6>>(a, st); }
void launch_y_210_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 14, 1>>(a, st); }
void launch_y_210_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 15, 1>>(a, st); }
void launch_y_210_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 5, 6>>(a, st); }
void launch_y_320_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 5, 8>>(a, st); }
void launch_y_320_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 8, 8>>(a, st); }
void launch_y_320_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 4, 8>>(a, st); }
void launch_y_450_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 9>>(a, st); }
void launch_y_450_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 5, 10>>(a, st); }
void launch_y_450_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 9, 10>>(a, st); }
void launch_y_648_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 8, 9>>(a, st); }
void launch_y_648_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 9, 9>>(a, st); }
void launch_y_648_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 6, 9>>(a, st); }
void launch_y_882_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 9>>(a, st); }
void launch_y_882_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 7, 14>>(a, st); }
void launch_y_882_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 9, 14>>(a, st); }
void launch_y_1176_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 12>>(a, st); }
void launch_y_1176_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 7, 14>>(a, st); }
void launch_y_1176_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 12, 14>>(a, st); }
void launch_y_1575_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 7, 15>>(a, st); }
void launch_y_1575_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 15, 15>>(a, st); }
void launch_y_2240_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 10, 14>>(a, st); }
void launch_y_2240_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 10, 16>>(a, st); }
void launch_y_2240_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 14, 16>>(a, st); }
}  // namespace dwcu
