// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_15(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<5, 3, 1>, 16>(a, st); }
void launch_x_48(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 6, 1>, 8>(a, st); }
void launch_x_98(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 1>, 8>(a, st); }
void launch_x_168(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 12, 1>, 8>(a, st); }
void launch_x_256(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 16, 1>, 4>(a, st); }
void launch_x_392(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 7, 7>, 2>(a, st); }
void launch_x_560(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 7, 8>, 2>(a, st); }
void launch_x_756(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 7, 9>, 2>(a, st); }
void launch_x_1024(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 8, 8>, 2>(a, st); }
void launch_x_1400(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 10, 10>, 1>(a, st); }
void launch_x_1920(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 10, 12>, 1>(a, st); }
}  // namespace dwcu
