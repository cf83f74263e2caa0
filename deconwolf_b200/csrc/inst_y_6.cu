// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_8_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 2, 1>>(a, st); }
void launch_y_8_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<2, 4, 1>>(a, st); }
void launch_y_8_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 1, 1>>(a, st); }
void launch_y_35_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 5, 1>>(a, st); }
void launch_y_35_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 7, 1>>(a, st); }
void launch_y_80_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 8, 1>>(a, st); }
void launch_y_80_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 10, 1>>(a, st); }
void launch_y_80_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 5, 1>>(a, st); }
void launch_y_144_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 12, 1>>(a, st); }
void launch_y_144_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 9, 1>>(a, st); }
void launch_y_144_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 16, 1>>(a, st); }
void launch_y_240_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 15, 1>>(a, st); }
void launch_y_240_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 16, 1>>(a, st); }
void launch_y_240_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 5, 6>>(a, st); }
void launch_y_350_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 7>>(a, st); }
void launch_y_350_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 5, 10>>(a, st); }
void launch_y_350_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 7, 10>>(a, st); }
void launch_y_500_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 10>>(a, st); }
void launch_y_500_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 10, 10>>(a, st); }
void launch_y_700_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 10>>(a, st); }
void launch_y_700_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 10, 10>>(a, st); }
void launch_y_700_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 5, 10>>(a, st); }
void launch_y_960_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 8, 10>>(a, st); }
void launch_y_960_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 8, 12>>(a, st); }
void launch_y_960_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 10, 12>>(a, st); }
void launch_y_1280_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 10>>(a, st); }
void launch_y_1280_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 8, 16>>(a, st); }
void launch_y_1280_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 10, 16>>(a, st); }
void launch_y_1728_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 12, 12>>(a, st); }
void launch_y_1728_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 9, 12>>(a, st); }
void launch_y_1728_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 12, 16>>(a, st); }
void launch_y_2400_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 10, 15>>(a, st); }
void launch_y_2400_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 10, 16>>(a, st); }
void launch_y_2400_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 15, 16>>(a, st); }
}  // namespace dwcu
