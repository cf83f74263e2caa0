// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_10_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 2, 1>>(a, st); }
void launch_y_10_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<2, 5, 1>>(a, st); }
void launch_y_10_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 1, 1>>(a, st); }
void launch_y_40_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 5, 1>>(a, st); }
void launch_y_40_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 8, 1>>(a, st); }
void launch_y_40_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 4, 1>>(a, st); }
void launch_y_84_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 7, 1>>(a, st); }
void launch_y_84_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 12, 1>>(a, st); }
void launch_y_84_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 6, 1>>(a, st); }
void launch_y_150_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 10, 1>>(a, st); }
void launch_y_150_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 15, 1>>(a, st); }
void launch_y_150_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 5, 5>>(a, st); }
void launch_y_245_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 5, 7>>(a, st); }
void launch_y_245_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 7, 7>>(a, st); }
void launch_y_375_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 5, 5>>(a, st); }
void launch_y_375_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 5, 15>>(a, st); }
void launch_y_512_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 8, 8>>(a, st); }
void launch_y_512_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 4, 8>>(a, st); }
void launch_y_512_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 8, 16>>(a, st); }
void launch_y_729_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 9, 9>>(a, st); }
void launch_y_980_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 10>>(a, st); }
void launch_y_980_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 14>>(a, st); }
void launch_y_980_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 10, 14>>(a, st); }
void launch_y_1344_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 12>>(a, st); }
void launch_y_1344_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 8, 14>>(a, st); }
void launch_y_1344_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 12, 14>>(a, st); }
void launch_y_1792_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 14>>(a, st); }
void launch_y_1792_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 16>>(a, st); }
void launch_y_1792_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 14, 16>>(a, st); }
void launch_y_2560_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 10, 16>>(a, st); }
void launch_y_2560_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 16, 16>>(a, st); }
}  // namespace dwcu
