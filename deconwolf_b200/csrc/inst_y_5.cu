// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_7(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 1, 1>>(a, st); }
void launch_y_32(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 4, 1>>(a, st); }
void launch_y_75(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 5, 1>>(a, st); }
void launch_y_140(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 10, 1>>(a, st); }
void launch_y_225(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 15, 1>>(a, st); }
void launch_y_343(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 7, 7>>(a, st); }
void launch_y_490(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 7, 7>>(a, st); }
void launch_y_686(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 7>>(a, st); }
void launch_y_945(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 7, 9>>(a, st); }
void launch_y_1260(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 9, 10>>(a, st); }
void launch_y_1680(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 10, 12>>(a, st); }
void launch_y_2352(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 12, 14>>(a, st); }
}  // namespace dwcu
