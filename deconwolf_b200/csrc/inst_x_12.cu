// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_x_16(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<4, 4, 1>, 8>(a, nb, st); }
void launch_x_49(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<7, 7, 1>, 8>(a, nb, st); }
void launch_x_100(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<10, 10, 1>, 8>(a, nb, st); }
void launch_x_175(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<7, 5, 5>, 8>(a, nb, st); }
void launch_x_270(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<9, 5, 6>, 8>(a, nb, st); }
void launch_x_400(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<10, 5, 8>, 4>(a, nb, st); }
void launch_x_567(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<9, 7, 9>, 4>(a, nb, st); }
void launch_x_768(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<12, 8, 8>, 4>(a, nb, st); }
void launch_x_1050(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<15, 7, 10>, 2>(a, nb, st); }
void launch_x_1440(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<12, 10, 12>, 2>(a, nb, st); }
void launch_x_1960(const XArgs &a, int nb, cudaStream_t st) { launch_x_t<Rad<14, 10, 14>, 2>(a, nb, st); }
}  // namespace dwcu
