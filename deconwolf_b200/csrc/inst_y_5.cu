// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_7_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 1, 1>>(a, st); }
void launch_y_32_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 4, 1>>(a, st); }
void launch_y_32_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 8, 1>>(a, st); }
void launch_y_32_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 2, 1>>(a, st); }
void launch_y_75_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 5, 1>>(a, st); }
void launch_y_75_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 15, 1>>(a, st); }
void launch_y_75_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 5, 5>>(a, st); }
void launch_y_140_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 10, 1>>(a, st); }
void launch_y_140_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 14, 1>>(a, st); }
void launch_y_140_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 4, 5>>(a, st); }
void launch_y_225_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 15, 1>>(a, st); }
void launch_y_225_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 5, 5>>(a, st); }
void launch_y_225_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 5, 9>>(a, st); }
void launch_y_343_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 7, 7>>(a, st); }
void launch_y_490_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 7>>(a, st); }
void launch_y_490_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 7, 10>>(a, st); }
void launch_y_490_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 5, 7>>(a, st); }
void launch_y_686_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 7>>(a, st); }
void launch_y_686_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 7, 14>>(a, st); }
void launch_y_945_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 7, 9>>(a, st); }
void launch_y_945_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 7, 15>>(a, st); }
void launch_y_945_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 9, 15>>(a, st); }
void launch_y_1260_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 9, 10>>(a, st); }
void launch_y_1260_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 9, 14>>(a, st); }
void launch_y_1260_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 10, 14>>(a, st); }
void launch_y_1680_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 10, 12>>(a, st); }
void launch_y_1680_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 10, 14>>(a, st); }
void launch_y_1680_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 12, 14>>(a, st); }
void launch_y_2352_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 12, 14>>(a, st); }
void launch_y_2352_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 14, 14>>(a, st); }
}  // namespace dwcu
