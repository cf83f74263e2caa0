// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_8(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<4, 2, 1>, 16>(a, st); }
void launch_x_35(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 5, 1>, 16>(a, st); }
void launch_x_80(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 8, 1>, 8>(a, st); }
void launch_x_144(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 12, 1>, 8>(a, st); }
void launch_x_240(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 15, 1>, 4>(a, st); }
void launch_x_350(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 7>, 2>(a, st); }
void launch_x_500(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 10>, 2>(a, st); }
void launch_x_700(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 7, 10>, 2>(a, st); }
void launch_x_960(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 8, 10>, 2>(a, st); }
void launch_x_1280(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 8, 10>, 1>(a, st); }
void launch_x_1728(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 12, 12>, 1>(a, st); }
}  // namespace dwcu
