// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_7(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 1, 1>, 16>(a, st); }
void launch_x_32(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 4, 1>, 8>(a, st); }
void launch_x_75(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 5, 1>, 8>(a, st); }
void launch_x_140(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 10, 1>, 8>(a, st); }
void launch_x_225(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 15, 1>, 8>(a, st); }
void launch_x_343(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 7, 7>, 2>(a, st); }
void launch_x_490(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 7, 7>, 2>(a, st); }
void launch_x_686(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 7>, 2>(a, st); }
void launch_x_945(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 7, 9>, 2>(a, st); }
void launch_x_1260(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 9, 10>, 1>(a, st); }
void launch_x_1680(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 10, 12>, 1>(a, st); }
}  // namespace dwcu
