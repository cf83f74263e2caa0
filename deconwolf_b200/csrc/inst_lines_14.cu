// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_18_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 3, 1>, 16>(a, nb, st); }
void launch_lines_18_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 6, 1>, 16>(a, nb, st); }
void launch_lines_18_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 3, 1>, 8>(a, nb, st); }
void launch_lines_50_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 1>, 16>(a, nb, st); }
void launch_lines_50_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 10, 1>, 16>(a, nb, st); }
void launch_lines_50_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 1>, 8>(a, nb, st); }
void launch_lines_105_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 1>, 16>(a, nb, st); }
void launch_lines_105_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 15, 1>, 16>(a, nb, st); }
void launch_lines_105_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 1>, 8>(a, nb, st); }
void launch_lines_180_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 1>, 16>(a, nb, st); }
void launch_lines_180_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 15, 1>, 16>(a, nb, st); }
void launch_lines_180_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 1>, 8>(a, nb, st); }
void launch_lines_280_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 7>, 16>(a, nb, st); }
void launch_lines_280_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 8>, 16>(a, nb, st); }
void launch_lines_280_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 7>, 8>(a, nb, st); }
void launch_lines_405_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 9>, 8>(a, nb, st); }
void launch_lines_405_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 9, 9>, 8>(a, nb, st); }
void launch_lines_405_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 9>, 4>(a, nb, st); }
void launch_lines_576_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 8, 8>, 8>(a, nb, st); }
void launch_lines_576_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 8, 9>, 8>(a, nb, st); }
void launch_lines_576_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 8, 8>, 4>(a, nb, st); }
void launch_lines_784_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 8>, 8>(a, nb, st); }
void launch_lines_784_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 14>, 8>(a, nb, st); }
void launch_lines_784_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 8>, 4>(a, nb, st); }
void launch_lines_1080_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 10>, 8>(a, nb, st); }
void launch_lines_1080_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 9, 12>, 8>(a, nb, st); }
void launch_lines_1080_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 10>, 4>(a, nb, st); }
void launch_lines_1470_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 14>, 4>(a, nb, st); }
void launch_lines_1470_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 15>, 4>(a, nb, st); }
void launch_lines_1470_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 14>, 2>(a, nb, st); }
void launch_lines_2016_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 12, 12>, 4>(a, nb, st); }
void launch_lines_2016_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 12, 14>, 4>(a, nb, st); }
void launch_lines_2016_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 12, 12>, 2>(a, nb, st); }
void launch_lines_2940_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 14, 14>, 4>(a, nb, st); }
void launch_lines_2940_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 14, 15>, 4>(a, nb, st); }
void launch_lines_2940_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 14, 14>, 2>(a, nb, st); }
}  // namespace dwcu
