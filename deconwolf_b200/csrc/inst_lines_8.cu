// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_9_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 3, 1>, 16>(a, nb, st); }
void launch_lines_9_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 1, 1>, 16>(a, nb, st); }
void launch_lines_9_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 3, 1>, 8>(a, nb, st); }
void launch_lines_36_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 6, 1>, 16>(a, nb, st); }
void launch_lines_36_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 4, 1>, 16>(a, nb, st); }
void launch_lines_36_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 6, 1>, 8>(a, nb, st); }
void launch_lines_81_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 9, 1>, 16>(a, nb, st); }
void launch_lines_81_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 3, 9>, 16>(a, nb, st); }
void launch_lines_81_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 9, 1>, 8>(a, nb, st); }
void launch_lines_147_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 3, 7>, 16>(a, nb, st); }
void launch_lines_147_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 7, 7>, 16>(a, nb, st); }
void launch_lines_147_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 3, 7>, 8>(a, nb, st); }
void launch_lines_243_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 3, 9>, 8>(a, nb, st); }
void launch_lines_243_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 9, 9>, 8>(a, nb, st); }
void launch_lines_243_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 3, 9>, 4>(a, nb, st); }
void launch_lines_360_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 6>, 16>(a, nb, st); }
void launch_lines_360_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 6, 10>, 16>(a, nb, st); }
void launch_lines_360_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 6>, 8>(a, nb, st); }
void launch_lines_504_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 8>, 8>(a, nb, st); }
void launch_lines_504_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 9>, 8>(a, nb, st); }
void launch_lines_504_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 8>, 4>(a, nb, st); }
void launch_lines_720_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 9>, 8>(a, nb, st); }
void launch_lines_720_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 8, 10>, 8>(a, nb, st); }
void launch_lines_720_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 9>, 4>(a, nb, st); }
void launch_lines_972_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 9>, 8>(a, nb, st); }
void launch_lines_972_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 9, 12>, 8>(a, nb, st); }
void launch_lines_972_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 9>, 4>(a, nb, st); }
void launch_lines_1296_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 12>, 4>(a, nb, st); }
void launch_lines_1296_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 12, 12>, 4>(a, nb, st); }
void launch_lines_1296_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 12>, 2>(a, nb, st); }
void launch_lines_1764_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 14>, 4>(a, nb, st); }
void launch_lines_1764_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 14, 14>, 4>(a, nb, st); }
void launch_lines_1764_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 14>, 2>(a, nb, st); }
void launch_lines_2520_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 14>, 4>(a, nb, st); }
void launch_lines_2520_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 12, 15>, 4>(a, nb, st); }
void launch_lines_2520_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 14>, 2>(a, nb, st); }
}  // namespace dwcu
