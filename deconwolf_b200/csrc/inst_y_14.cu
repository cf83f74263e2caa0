// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_20(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 4, 1>>(a, st); }
void launch_y_54(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 6, 1>>(a, st); }
void launch_y_108(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 9, 1>>(a, st); }
void launch_y_189(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 3, 7>>(a, st); }
void launch_y_288(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 6, 6>>(a, st); }
void launch_y_420(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 6, 7>>(a, st); }
void launch_y_588(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 7, 7>>(a, st); }
void launch_y_800(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 8, 10>>(a, st); }
void launch_y_1120(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 10>>(a, st); }
void launch_y_1500(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 10, 10>>(a, st); }
void launch_y_2025(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 9, 15>>(a, st); }
void launch_y_3072(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 12, 16>>(a, st); }
}  // namespace dwcu
