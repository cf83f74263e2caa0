// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_9(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<3, 3, 1>, 32>(a, st); }
void launch_x_36(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<6, 6, 1>, 16>(a, st); }
void launch_x_81(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 9, 1>, 8>(a, st); }
void launch_x_147(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 3, 7>, 2>(a, st); }
void launch_x_243(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 3, 9>, 2>(a, st); }
void launch_x_360(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 6, 6>, 2>(a, st); }
void launch_x_504(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 7, 8>, 2>(a, st); }
void launch_x_720(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 8, 9>, 2>(a, st); }
void launch_x_972(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 9, 9>, 2>(a, st); }
void launch_x_1296(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 9, 12>, 1>(a, st); }
void launch_x_1764(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 9, 14>, 1>(a, st); }
}  // namespace dwcu
