// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_15(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 3, 1>>(a, st); }
void launch_y_48(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 6, 1>>(a, st); }
void launch_y_98(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 1>>(a, st); }
void launch_y_168(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 12, 1>>(a, st); }
void launch_y_256(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 16, 1>>(a, st); }
void launch_y_392(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 7, 7>>(a, st); }
void launch_y_560(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 8>>(a, st); }
void launch_y_756(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 7, 9>>(a, st); }
void launch_y_1024(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 8>>(a, st); }
void launch_y_1400(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 10, 10>>(a, st); }
void launch_y_1920(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 10, 12>>(a, st); }
void launch_y_2744(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 14, 14>>(a, st); }
}  // namespace dwcu
