// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_20(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<5, 4, 1>, 16>(a, st); }
void launch_x_54(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 6, 1>, 8>(a, st); }
void launch_x_108(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 9, 1>, 8>(a, st); }
void launch_x_189(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 3, 7>, 2>(a, st); }
void launch_x_288(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 6, 6>, 2>(a, st); }
void launch_x_420(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 6, 7>, 2>(a, st); }
void launch_x_588(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 7, 7>, 2>(a, st); }
void launch_x_800(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 8, 10>, 2>(a, st); }
void launch_x_1120(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 8, 10>, 2>(a, st); }
void launch_x_1500(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 10, 10>, 1>(a, st); }
void launch_x_2025(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 9, 15>, 1>(a, st); }
}  // namespace dwcu
