// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_6(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 2, 1>>(a, st); }
void launch_y_30(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 5, 1>>(a, st); }
void launch_y_72(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 8, 1>>(a, st); }
void launch_y_135(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 9, 1>>(a, st); }
void launch_y_224(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 14, 1>>(a, st); }
void launch_y_336(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 6, 7>>(a, st); }
void launch_y_486(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 6, 9>>(a, st); }
void launch_y_675(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 5, 9>>(a, st); }
void launch_y_900(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 9, 10>>(a, st); }
void launch_y_1215(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 9, 9>>(a, st); }
void launch_y_1620(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 9, 12>>(a, st); }
void launch_y_2304(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 12, 12>>(a, st); }
}  // namespace dwcu
