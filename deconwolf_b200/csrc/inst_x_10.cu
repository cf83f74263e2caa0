// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_14(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 2, 1>, 16>(a, st); }
void launch_x_45(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 5, 1>, 8>(a, st); }
void launch_x_96(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<12, 8, 1>, 8>(a, st); }
void launch_x_162(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<9, 3, 6>, 2>(a, st); }
void launch_x_252(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<7, 6, 6>, 2>(a, st); }
void launch_x_384(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<8, 6, 8>, 2>(a, st); }
void launch_x_540(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<10, 6, 9>, 2>(a, st); }
void launch_x_750(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 5, 10>, 2>(a, st); }
void launch_x_1008(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 8, 9>, 2>(a, st); }
void launch_x_1372(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<14, 7, 14>, 1>(a, st); }
void launch_x_1890(const XArgs &a, cudaStream_t st) { launch_x_t<Rad<15, 9, 14>, 1>(a, st); }
}  // namespace dwcu
