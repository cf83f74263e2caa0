// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<2, 1, 1>>(a, st); }
void launch_y_24(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 4, 1>>(a, st); }
void launch_y_60(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 6, 1>>(a, st); }
void launch_y_120(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 10, 1>>(a, st); }
void launch_y_196(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 14, 1>>(a, st); }
void launch_y_300(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 6>>(a, st); }
void launch_y_441(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 7, 7>>(a, st); }
void launch_y_630(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 9>>(a, st); }
void launch_y_840(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 7, 10>>(a, st); }
void launch_y_1134(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 9, 9>>(a, st); }
void launch_y_1536(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 12>>(a, st); }
void launch_y_2100(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 10, 14>>(a, st); }
void launch_y_3150(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 14, 15>>(a, st); }
}  // namespace dwcu
