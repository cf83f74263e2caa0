// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_14(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 2, 1>>(a, st); }
void launch_y_45(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 5, 1>>(a, st); }
void launch_y_96(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 8, 1>>(a, st); }
void launch_y_162(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 3, 6>>(a, st); }
void launch_y_252(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 6, 6>>(a, st); }
void launch_y_384(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 6, 8>>(a, st); }
void launch_y_540(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 6, 9>>(a, st); }
void launch_y_750(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 5, 10>>(a, st); }
void launch_y_1008(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 9>>(a, st); }
void launch_y_1372(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 14>>(a, st); }
void launch_y_1890(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 9, 14>>(a, st); }
void launch_y_2700(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 12, 15>>(a, st); }
}  // namespace dwcu
