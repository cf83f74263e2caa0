// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_9(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 3, 1>>(a, st); }
void launch_y_36(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 6, 1>>(a, st); }
void launch_y_81(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 9, 1>>(a, st); }
void launch_y_147(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 3, 7>>(a, st); }
void launch_y_243(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 3, 9>>(a, st); }
void launch_y_360(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 6, 6>>(a, st); }
void launch_y_504(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 7, 8>>(a, st); }
void launch_y_720(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 8, 9>>(a, st); }
void launch_y_972(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 9, 9>>(a, st); }
void launch_y_1296(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 9, 12>>(a, st); }
void launch_y_1764(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 9, 14>>(a, st); }
void launch_y_2520(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 12, 14>>(a, st); }
}  // namespace dwcu
