// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_3_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 1, 1>, 16>(a, nb, st); }
void launch_lines_3_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 1, 1>, 8>(a, nb, st); }
void launch_lines_25_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 5, 1>, 16>(a, nb, st); }
void launch_lines_25_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 5, 1>, 8>(a, nb, st); }
void launch_lines_63_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 1>, 16>(a, nb, st); }
void launch_lines_63_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 9, 1>, 16>(a, nb, st); }
void launch_lines_63_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 1>, 8>(a, nb, st); }
void launch_lines_125_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 5, 5>, 16>(a, nb, st); }
void launch_lines_125_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 5, 5>, 8>(a, nb, st); }
void launch_lines_200_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 5>, 16>(a, nb, st); }
void launch_lines_200_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 5, 8>, 16>(a, nb, st); }
void launch_lines_200_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 5>, 8>(a, nb, st); }
void launch_lines_315_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 7>, 16>(a, nb, st); }
void launch_lines_315_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 9>, 16>(a, nb, st); }
void launch_lines_315_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 7>, 8>(a, nb, st); }
void launch_lines_448_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 8>, 16>(a, nb, st); }
void launch_lines_448_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 8, 8>, 16>(a, nb, st); }
void launch_lines_448_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 8>, 8>(a, nb, st); }
void launch_lines_640_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 8>, 8>(a, nb, st); }
void launch_lines_640_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 8, 10>, 8>(a, nb, st); }
void launch_lines_640_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 8>, 4>(a, nb, st); }
void launch_lines_864_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 9>, 8>(a, nb, st); }
void launch_lines_864_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 8, 12>, 8>(a, nb, st); }
void launch_lines_864_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 9>, 4>(a, nb, st); }
void launch_lines_1152_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 12>, 4>(a, nb, st); }
void launch_lines_1152_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 12, 12>, 4>(a, nb, st); }
void launch_lines_1152_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 12>, 2>(a, nb, st); }
void launch_lines_1568_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 14>, 4>(a, nb, st); }
void launch_lines_1568_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 14, 14>, 4>(a, nb, st); }
void launch_lines_1568_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 14>, 2>(a, nb, st); }
void launch_lines_2160_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 12>, 4>(a, nb, st); }
void launch_lines_2160_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 12, 15>, 4>(a, nb, st); }
void launch_lines_2160_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 12>, 2>(a, nb, st); }
void launch_lines_3360_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 14, 15>, 2>(a, nb, st); }
void launch_lines_3360_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 14, 16>, 2>(a, nb, st); }
}  // namespace dwcu
