// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_3(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<3, 1, 1>, 32>(a, st); }
void launch_x_25(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<5, 5, 1>, 16>(a, st); }
void launch_x_63(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 7, 1>, 8>(a, st); }
void launch_x_125(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<5, 5, 5>, 4>(a, st); }
void launch_x_200(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 5, 5>, 2>(a, st); }
void launch_x_315(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 5, 7>, 2>(a, st); }
void launch_x_448(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 7, 8>, 2>(a, st); }
void launch_x_640(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 8, 8>, 2>(a, st); }
void launch_x_864(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 8, 9>, 2>(a, st); }
void launch_x_1152(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 8, 12>, 1>(a, st); }
void launch_x_1568(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 8, 14>, 1>(a, st); }
}  // namespace dwcu
