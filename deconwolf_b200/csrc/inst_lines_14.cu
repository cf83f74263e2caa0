// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_18(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 3, 1>, 16>(a, nb, st); }
void launch_lines_50(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 1>, 16>(a, nb, st); }
void launch_lines_105(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 1>, 16>(a, nb, st); }
void launch_lines_180(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 1>, 16>(a, nb, st); }
void launch_lines_280(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 7>, 16>(a, nb, st); }
void launch_lines_405(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 9>, 8>(a, nb, st); }
void launch_lines_576(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 8, 8>, 8>(a, nb, st); }
void launch_lines_784(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 8>, 8>(a, nb, st); }
void launch_lines_1080(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 10>, 8>(a, nb, st); }
void launch_lines_1470(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 14>, 4>(a, nb, st); }
void launch_lines_2016(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 12, 12>, 4>(a, nb, st); }
void launch_lines_2940(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 14, 14>, 4>(a, nb, st); }
}  // namespace dwcu
