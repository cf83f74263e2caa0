// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_16(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 4, 1>, 16>(a, nb, st); }
void launch_lines_49(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 7, 1>, 16>(a, nb, st); }
void launch_lines_100(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 10, 1>, 16>(a, nb, st); }
void launch_lines_175(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 5>, 16>(a, nb, st); }
void launch_lines_270(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 6>, 16>(a, nb, st); }
void launch_lines_400(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 8>, 8>(a, nb, st); }
void launch_lines_567(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 9>, 8>(a, nb, st); }
void launch_lines_768(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 8>, 8>(a, nb, st); }
void launch_lines_1050(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 10>, 4>(a, nb, st); }
void launch_lines_1440(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 10, 12>, 4>(a, nb, st); }
void launch_lines_1960(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 14>, 4>(a, nb, st); }
void launch_lines_2880(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 15>, 4>(a, nb, st); }
}  // namespace dwcu
