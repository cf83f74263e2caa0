// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_20_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 4, 1>>(a, st); }
void launch_y_20_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 5, 1>>(a, st); }
void launch_y_20_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 2, 1>>(a, st); }
void launch_y_54_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 6, 1>>(a, st); }
void launch_y_54_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 9, 1>>(a, st); }
void launch_y_54_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 3, 6>>(a, st); }
void launch_y_108_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 9, 1>>(a, st); }
void launch_y_108_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 12, 1>>(a, st); }
void launch_y_108_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 3, 6>>(a, st); }
void launch_y_189_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 3, 7>>(a, st); }
void launch_y_189_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 3, 9>>(a, st); }
void launch_y_189_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 7, 9>>(a, st); }
void launch_y_288_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 6, 6>>(a, st); }
void launch_y_288_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 6, 8>>(a, st); }
void launch_y_288_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 4, 8>>(a, st); }
void launch_y_420_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 6, 7>>(a, st); }
void launch_y_420_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 6, 10>>(a, st); }
void launch_y_420_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 7, 10>>(a, st); }
void launch_y_588_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 7, 7>>(a, st); }
void launch_y_588_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 7, 12>>(a, st); }
void launch_y_588_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 6, 7>>(a, st); }
void launch_y_800_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 8, 10>>(a, st); }
void launch_y_800_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 10, 10>>(a, st); }
void launch_y_800_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 5, 10>>(a, st); }
void launch_y_1120_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 10>>(a, st); }
void launch_y_1120_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 8, 14>>(a, st); }
void launch_y_1120_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 10, 14>>(a, st); }
void launch_y_1500_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 10, 10>>(a, st); }
void launch_y_1500_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 10, 15>>(a, st); }
void launch_y_2025_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 9, 15>>(a, st); }
void launch_y_2025_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 15, 15>>(a, st); }
void launch_y_3072_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 12, 16>>(a, st); }
void launch_y_3072_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 16, 16>>(a, st); }
}  // namespace dwcu
