// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_18(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 3, 1>>(a, st); }
void launch_y_50(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 1>>(a, st); }
void launch_y_105(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 7, 1>>(a, st); }
void launch_y_180(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 12, 1>>(a, st); }
void launch_y_280(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 5, 7>>(a, st); }
void launch_y_405(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 5, 9>>(a, st); }
void launch_y_576(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 8, 8>>(a, st); }
void launch_y_784(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 8>>(a, st); }
void launch_y_1080(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 9, 10>>(a, st); }
void launch_y_1470(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 7, 14>>(a, st); }
void launch_y_2016(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 12, 12>>(a, st); }
void launch_y_2940(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 14, 14>>(a, st); }
}  // namespace dwcu
