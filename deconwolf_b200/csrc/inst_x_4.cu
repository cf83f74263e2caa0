// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_6(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<3, 2, 1>, 32>(a, st); }
void launch_x_30(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<6, 5, 1>, 16>(a, st); }
void launch_x_72(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 8, 1>, 8>(a, st); }
void launch_x_135(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 9, 1>, 8>(a, st); }
void launch_x_224(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 14, 1>, 4>(a, st); }
void launch_x_336(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 6, 7>, 2>(a, st); }
void launch_x_486(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 6, 9>, 2>(a, st); }
void launch_x_675(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 5, 9>, 2>(a, st); }
void launch_x_900(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 9, 10>, 2>(a, st); }
void launch_x_1215(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 9, 9>, 1>(a, st); }
void launch_x_1620(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 9, 12>, 1>(a, st); }
}  // namespace dwcu
