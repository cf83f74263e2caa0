// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_12(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<4, 3, 1>, 16>(a, st); }
void launch_x_42(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 6, 1>, 16>(a, st); }
void launch_x_90(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 9, 1>, 8>(a, st); }
void launch_x_160(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 10, 1>, 4>(a, st); }
void launch_x_250(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 5>, 2>(a, st); }
void launch_x_378(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 6, 7>, 2>(a, st); }
void launch_x_525(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 5, 7>, 2>(a, st); }
void launch_x_735(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 7, 7>, 2>(a, st); }
void launch_x_1000(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 10, 10>, 2>(a, st); }
void launch_x_1350(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 9, 10>, 1>(a, st); }
void launch_x_1800(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 10, 12>, 1>(a, st); }
}  // namespace dwcu
