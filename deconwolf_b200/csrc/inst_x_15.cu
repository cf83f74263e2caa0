// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_21(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 3, 1>, 16>(a, st); }
void launch_x_56(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 7, 1>, 8>(a, st); }
void launch_x_112(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 8, 1>, 8>(a, st); }
void launch_x_192(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 12, 1>, 4>(a, st); }
void launch_x_294(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 6, 7>, 2>(a, st); }
void launch_x_432(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 6, 8>, 2>(a, st); }
void launch_x_600(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 6, 10>, 2>(a, st); }
void launch_x_810(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 9, 9>, 2>(a, st); }
void launch_x_1125(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 5, 15>, 1>(a, st); }
void launch_x_1512(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 9, 12>, 1>(a, st); }
void launch_x_2048(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 8, 16>, 1>(a, st); }
}  // namespace dwcu
