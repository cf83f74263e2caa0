// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_2_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<2, 1, 1>>(a, st); }
void launch_y_24_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 4, 1>>(a, st); }
void launch_y_24_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 6, 1>>(a, st); }
void launch_y_24_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 3, 1>>(a, st); }
void launch_y_60_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 6, 1>>(a, st); }
void launch_y_60_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 10, 1>>(a, st); }
void launch_y_60_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 5, 1>>(a, st); }
void launch_y_120_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 10, 1>>(a, st); }
void launch_y_120_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 12, 1>>(a, st); }
void launch_y_120_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 8, 1>>(a, st); }
void launch_y_196_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 14, 1>>(a, st); }
void launch_y_196_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 4, 7>>(a, st); }
void launch_y_196_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 7, 7>>(a, st); }
void launch_y_300_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 6>>(a, st); }
void launch_y_300_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 5, 10>>(a, st); }
void launch_y_300_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 6, 10>>(a, st); }
void launch_y_441_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 7, 7>>(a, st); }
void launch_y_441_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 7, 9>>(a, st); }
void launch_y_630_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 9>>(a, st); }
void launch_y_630_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 7, 10>>(a, st); }
void launch_y_630_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 9, 10>>(a, st); }
void launch_y_840_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 7, 10>>(a, st); }
void launch_y_840_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 12>>(a, st); }
void launch_y_840_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 10, 12>>(a, st); }
void launch_y_1134_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 9, 9>>(a, st); }
void launch_y_1134_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 9, 14>>(a, st); }
void launch_y_1536_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 12>>(a, st); }
void launch_y_1536_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 8, 16>>(a, st); }
void launch_y_1536_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 12, 16>>(a, st); }
void launch_y_2100_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 10, 14>>(a, st); }
void launch_y_2100_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 10, 15>>(a, st); }
void launch_y_2100_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 14, 15>>(a, st); }
void launch_y_3150_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 14, 15>>(a, st); }
void launch_y_3150_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 15, 15>>(a, st); }
}  // namespace dwcu
