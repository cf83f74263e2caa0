// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_18(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<6, 3, 1>, 8>(a, nb, st); }
void launch_x_50(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<10, 5, 1>, 8>(a, nb, st); }
void launch_x_105(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<15, 7, 1>, 8>(a, nb, st); }
void launch_x_180(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<15, 12, 1>, 8>(a, nb, st); }
void launch_x_280(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<8, 5, 7>, 8>(a, nb, st); }
void launch_x_405(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<9, 5, 9>, 4>(a, nb, st); }
void launch_x_576(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<9, 8, 8>, 4>(a, nb, st); }
void launch_x_784(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<14, 7, 8>, 4>(a, nb, st); }
void launch_x_1080(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<12, 9, 10>, 4>(a, nb, st); }
void launch_x_1470(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<15, 7, 14>, 2>(a, nb, st); }
void launch_x_2016(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<14, 12, 12>, 2>(a, nb, st); }
}  // namespace dwcu
