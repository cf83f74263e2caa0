// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_9(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 3, 1>, 16>(a, nb, st); }
void launch_lines_36(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 6, 1>, 16>(a, nb, st); }
void launch_lines_81(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 9, 1>, 16>(a, nb, st); }
void launch_lines_147(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 3, 7>, 16>(a, nb, st); }
void launch_lines_243(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 3, 9>, 8>(a, nb, st); }
void launch_lines_360(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 6>, 16>(a, nb, st); }
void launch_lines_504(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 8>, 8>(a, nb, st); }
void launch_lines_720(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 9>, 8>(a, nb, st); }
void launch_lines_972(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 9>, 8>(a, nb, st); }
void launch_lines_1296(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 12>, 4>(a, nb, st); }
void launch_lines_1764(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 14>, 4>(a, nb, st); }
void launch_lines_2520(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 14>, 4>(a, nb, st); }
}  // namespace dwcu
