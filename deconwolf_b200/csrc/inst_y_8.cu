// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_10(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 2, 1>>(a, st); }
void launch_y_40(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 5, 1>>(a, st); }
void launch_y_84(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 7, 1>>(a, st); }
void launch_y_150(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 10, 1>>(a, st); }
void launch_y_245(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 5, 7>>(a, st); }
void launch_y_375(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 5, 5>>(a, st); }
void launch_y_512(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 8, 8>>(a, st); }
void launch_y_729(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 9, 9>>(a, st); }
void launch_y_980(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 10>>(a, st); }
void launch_y_1344(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 12>>(a, st); }
void launch_y_1792(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 14>>(a, st); }
void launch_y_2560(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 10, 16>>(a, st); }
}  // namespace dwcu
