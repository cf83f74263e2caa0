// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_16(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 4, 1>>(a, st); }
void launch_y_49(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 7, 1>>(a, st); }
void launch_y_100(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 10, 1>>(a, st); }
void launch_y_175(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 5, 5>>(a, st); }
void launch_y_270(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 5, 6>>(a, st); }
void launch_y_400(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 8>>(a, st); }
void launch_y_567(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 7, 9>>(a, st); }
void launch_y_768(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 8, 8>>(a, st); }
void launch_y_1050(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 7, 10>>(a, st); }
void launch_y_1440(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 10, 12>>(a, st); }
void launch_y_1960(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 10, 14>>(a, st); }
void launch_y_2880(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 12, 15>>(a, st); }
}  // namespace dwcu
