// generated by gen_plans.py -- do not edit
#define DW_PAIRED_ADDS 0
#include "launch.cuh"
namespace dwcu {
void launch_y_3(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<3, 1, 1>>(a, st); }
void launch_y_25(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 5, 1>>(a, st); }
void launch_y_63(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 7, 1>>(a, st); }
void launch_y_125(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<5, 5, 5>>(a, st); }
void launch_y_200(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 5, 5>>(a, st); }
void launch_y_315(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<9, 5, 7>>(a, st); }
void launch_y_448(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<8, 7, 8>>(a, st); }
void launch_y_640(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<10, 8, 8>>(a, st); }
void launch_y_864(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 8, 9>>(a, st); }
void launch_y_1152(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<12, 8, 12>>(a, st); }
void launch_y_1568(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<14, 8, 14>>(a, st); }
void launch_y_2160(const YArgs &a, cudaStream_t st) { launch_y_t<Rad<15, 12, 12>>(a, st); }
}  // namespace dwcu
