// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_4(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<2, 2, 1>>(a, st); }
void launch_y_27(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 3, 1>>(a, st); }
void launch_y_64(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 8, 1>>(a, st); }
void launch_y_126(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 9, 1>>(a, st); }
void launch_y_210(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 14, 1>>(a, st); }
void launch_y_320(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 5, 8>>(a, st); }
void launch_y_450(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 5, 9>>(a, st); }
void launch_y_648(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 8, 9>>(a, st); }
void launch_y_882(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 9>>(a, st); }
void launch_y_1176(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 7, 12>>(a, st); }
void launch_y_1575(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 7, 15>>(a, st); }
void launch_y_2240(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 10, 14>>(a, st); }
}  // namespace dwcu
