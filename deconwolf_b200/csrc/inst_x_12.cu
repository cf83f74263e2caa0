// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_16(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<4, 4, 1>, 16>(a, st); }
void launch_x_49(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 7, 1>, 16>(a, st); }
void launch_x_100(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 10, 1>, 8>(a, st); }
void launch_x_175(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 5, 5>, 2>(a, st); }
void launch_x_270(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 5, 6>, 2>(a, st); }
void launch_x_400(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 5, 8>, 2>(a, st); }
void launch_x_567(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 7, 9>, 2>(a, st); }
void launch_x_768(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 8, 8>, 2>(a, st); }
void launch_x_1050(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 7, 10>, 2>(a, st); }
void launch_x_1440(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 10, 12>, 1>(a, st); }
void launch_x_1960(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 10, 14>, 1>(a, st); }
}  // namespace dwcu
