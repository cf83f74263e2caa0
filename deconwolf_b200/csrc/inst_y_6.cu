// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_8(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<4, 2, 1>>(a, st); }
void launch_y_35(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 5, 1>>(a, st); }
void launch_y_80(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 8, 1>>(a, st); }
void launch_y_144(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 12, 1>>(a, st); }
void launch_y_240(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 15, 1>>(a, st); }
void launch_y_350(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 7>>(a, st); }
void launch_y_500(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 10>>(a, st); }
void launch_y_700(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 10>>(a, st); }
void launch_y_960(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 8, 10>>(a, st); }
void launch_y_1280(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 10>>(a, st); }
void launch_y_1728(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 12, 12>>(a, st); }
void launch_y_2400(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 10, 15>>(a, st); }
}  // namespace dwcu
