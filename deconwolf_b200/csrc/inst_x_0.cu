// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_2(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<2, 1, 1>, 32>(a, st); }
void launch_x_24(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<6, 4, 1>, 16>(a, st); }
void launch_x_60(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 6, 1>, 8>(a, st); }
void launch_x_120(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 10, 1>, 8>(a, st); }
void launch_x_196(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 14, 1>, 8>(a, st); }
void launch_x_300(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 6>, 2>(a, st); }
void launch_x_441(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 7, 7>, 2>(a, st); }
void launch_x_630(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 7, 9>, 2>(a, st); }
void launch_x_840(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 7, 10>, 2>(a, st); }
void launch_x_1134(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 9, 9>, 2>(a, st); }
void launch_x_1536(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 8, 12>, 1>(a, st); }
}  // namespace dwcu
