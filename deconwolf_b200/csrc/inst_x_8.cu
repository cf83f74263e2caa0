// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_10(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<5, 2, 1>, 16>(a, st); }
void launch_x_40(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 5, 1>, 8>(a, st); }
void launch_x_84(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 7, 1>, 8>(a, st); }
void launch_x_150(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 10, 1>, 8>(a, st); }
void launch_x_245(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 5, 7>, 2>(a, st); }
void launch_x_375(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 5, 5>, 2>(a, st); }
void launch_x_512(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 8, 8>, 2>(a, st); }
void launch_x_729(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 9, 9>, 2>(a, st); }
void launch_x_980(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 10>, 2>(a, st); }
void launch_x_1344(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 8, 12>, 1>(a, st); }
void launch_x_1792(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<16, 8, 14>, 1>(a, st); }
}  // namespace dwcu
