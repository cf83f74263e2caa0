// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_12(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 3, 1>>(a, st); }
void launch_y_42(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 6, 1>>(a, st); }
void launch_y_90(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 9, 1>>(a, st); }
void launch_y_160(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 10, 1>>(a, st); }
void launch_y_250(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 5>>(a, st); }
void launch_y_378(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 6, 7>>(a, st); }
void launch_y_525(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 5, 7>>(a, st); }
void launch_y_735(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 7, 7>>(a, st); }
void launch_y_1000(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 10, 10>>(a, st); }
void launch_y_1350(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 9, 10>>(a, st); }
void launch_y_1800(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 10, 12>>(a, st); }
void launch_y_2688(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 12, 14>>(a, st); }
}  // namespace dwcu
