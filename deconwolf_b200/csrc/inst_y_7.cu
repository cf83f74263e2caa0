// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_9_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 3, 1>>(a, st); }
void launch_y_9_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 1, 1>>(a, st); }
void launch_y_36_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 6, 1>>(a, st); }
void launch_y_36_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 4, 1>>(a, st); }
void launch_y_36_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 9, 1>>(a, st); }
void launch_y_81_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 9, 1>>(a, st); }
void launch_y_81_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 3, 9>>(a, st); }
void launch_y_147_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 3, 7>>(a, st); }
void launch_y_147_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 7, 7>>(a, st); }
void launch_y_243_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 3, 9>>(a, st); }
void launch_y_243_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 9, 9>>(a, st); }
void launch_y_360_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 6, 6>>(a, st); }
void launch_y_360_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 6, 10>>(a, st); }
void launch_y_360_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 5, 8>>(a, st); }
void launch_y_504_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 7, 8>>(a, st); }
void launch_y_504_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 7, 9>>(a, st); }
void launch_y_504_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 8, 9>>(a, st); }
void launch_y_720_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 8, 9>>(a, st); }
void launch_y_720_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 8, 10>>(a, st); }
void launch_y_720_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 9, 10>>(a, st); }
void launch_y_972_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 9, 9>>(a, st); }
void launch_y_972_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 9, 12>>(a, st); }
void launch_y_1296_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 9, 12>>(a, st); }
void launch_y_1296_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 12, 12>>(a, st); }
void launch_y_1296_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 9, 9>>(a, st); }
void launch_y_1764_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 9, 14>>(a, st); }
void launch_y_1764_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 14, 14>>(a, st); }
void launch_y_2520_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 12, 14>>(a, st); }
void launch_y_2520_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 12, 15>>(a, st); }
void launch_y_2520_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 14, 15>>(a, st); }
}  // namespace dwcu
