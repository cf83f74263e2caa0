// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_21_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 3, 1>>(a, st); }
void launch_y_21_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 7, 1>>(a, st); }
void launch_y_56_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 7, 1>>(a, st); }
void launch_y_56_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 8, 1>>(a, st); }
void launch_y_56_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 4, 1>>(a, st); }
void launch_y_112_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 1>>(a, st); }
void launch_y_112_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 14, 1>>(a, st); }
void launch_y_112_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 7, 1>>(a, st); }
void launch_y_192_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 12, 1>>(a, st); }
void launch_y_192_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 16, 1>>(a, st); }
void launch_y_192_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 4, 6>>(a, st); }
void launch_y_294_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<7, 6, 7>>(a, st); }
void launch_y_294_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 7, 7>>(a, st); }
void launch_y_294_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 3, 7>>(a, st); }
void launch_y_432_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 6, 8>>(a, st); }
void launch_y_432_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 6, 9>>(a, st); }
void launch_y_432_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 8, 9>>(a, st); }
void launch_y_600_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 6, 10>>(a, st); }
void launch_y_600_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<6, 10, 10>>(a, st); }
void launch_y_600_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 5, 10>>(a, st); }
void launch_y_810_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 9, 9>>(a, st); }
void launch_y_810_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 9, 10>>(a, st); }
void launch_y_810_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 6, 9>>(a, st); }
void launch_y_1125_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 5, 15>>(a, st); }
void launch_y_1125_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 15, 15>>(a, st); }
void launch_y_1512_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 9, 12>>(a, st); }
void launch_y_1512_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 9, 14>>(a, st); }
void launch_y_1512_2(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 12, 14>>(a, st); }
void launch_y_2048_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 8, 16>>(a, st); }
void launch_y_2048_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 16, 16>>(a, st); }
void launch_y_3136_0(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<16, 14, 14>>(a, st); }
void launch_y_3136_1(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 14, 16>>(a, st); }
}  // namespace dwcu
