// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_21(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 3, 1>>(a, st); }
void launch_y_56(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 7, 1>>(a, st); }
void launch_y_112(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 1>>(a, st); }
void launch_y_192(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 12, 1>>(a, st); }
void launch_y_294(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 6, 7>>(a, st); }
void launch_y_432(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 6, 8>>(a, st); }
void launch_y_600(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 6, 10>>(a, st); }
void launch_y_810(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 9, 9>>(a, st); }
void launch_y_1125(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 5, 15>>(a, st); }
void launch_y_1512(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 9, 12>>(a, st); }
void launch_y_2048(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 16>>(a, st); }
void launch_y_3136(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 14, 14>>(a, st); }
}  // namespace dwcu
