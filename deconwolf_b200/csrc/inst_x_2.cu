// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_4(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<2, 2, 1>, 32>(a, st); }
void launch_x_27(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 3, 1>, 8>(a, st); }
void launch_x_64(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 8, 1>, 8>(a, st); }
void launch_x_126(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 9, 1>, 8>(a, st); }
void launch_x_210(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 14, 1>, 8>(a, st); }
void launch_x_320(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 5, 8>, 2>(a, st); }
void launch_x_450(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 9>, 2>(a, st); }
void launch_x_648(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 8, 9>, 2>(a, st); }
void launch_x_882(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 9>, 2>(a, st); }
void launch_x_1176(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 12>, 1>(a, st); }
void launch_x_1575(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 7, 15>, 1>(a, st); }
}  // namespace dwcu
