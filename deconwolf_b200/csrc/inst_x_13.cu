// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_18(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<6, 3, 1>, 16>(a, st); }
void launch_x_50(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 1>, 8>(a, st); }
void launch_x_105(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 7, 1>, 8>(a, st); }
void launch_x_180(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 12, 1>, 8>(a, st); }
void launch_x_280(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 5, 7>, 2>(a, st); }
void launch_x_405(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 5, 9>, 2>(a, st); }
void launch_x_576(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 8, 8>, 2>(a, st); }
void launch_x_784(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 8>, 2>(a, st); }
void launch_x_1080(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 9, 10>, 2>(a, st); }
void launch_x_1470(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 7, 14>, 1>(a, st); }
void launch_x_2016(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 12, 12>, 1>(a, st); }
}  // namespace dwcu
