// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_7_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 1, 1>, 16>(a, nb, st); }
void launch_lines_7_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 1, 1>, 8>(a, nb, st); }
void launch_lines_32_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 4, 1>, 16>(a, nb, st); }
void launch_lines_32_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 8, 1>, 16>(a, nb, st); }
void launch_lines_32_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 4, 1>, 8>(a, nb, st); }
void launch_lines_75_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 1>, 16>(a, nb, st); }
void launch_lines_75_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 15, 1>, 16>(a, nb, st); }
void launch_lines_75_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 1>, 8>(a, nb, st); }
void launch_lines_140_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 1>, 16>(a, nb, st); }
void launch_lines_140_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 14, 1>, 16>(a, nb, st); }
void launch_lines_140_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 1>, 8>(a, nb, st); }
void launch_lines_225_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 15, 1>, 16>(a, nb, st); }
void launch_lines_225_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 5>, 16>(a, nb, st); }
void launch_lines_225_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 15, 1>, 8>(a, nb, st); }
void launch_lines_343_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 7, 7>, 16>(a, nb, st); }
void launch_lines_343_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 7, 7>, 8>(a, nb, st); }
void launch_lines_490_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 7>, 8>(a, nb, st); }
void launch_lines_490_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 7, 10>, 8>(a, nb, st); }
void launch_lines_490_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 7>, 4>(a, nb, st); }
void launch_lines_686_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 7>, 8>(a, nb, st); }
void launch_lines_686_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 7, 14>, 8>(a, nb, st); }
void launch_lines_686_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 7>, 4>(a, nb, st); }
void launch_lines_945_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 9>, 4>(a, nb, st); }
void launch_lines_945_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 15>, 4>(a, nb, st); }
void launch_lines_945_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 9>, 2>(a, nb, st); }
void launch_lines_1260_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 10>, 4>(a, nb, st); }
void launch_lines_1260_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 9, 14>, 4>(a, nb, st); }
void launch_lines_1260_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 10>, 2>(a, nb, st); }
void launch_lines_1680_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 12>, 4>(a, nb, st); }
void launch_lines_1680_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 10, 14>, 4>(a, nb, st); }
void launch_lines_1680_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 12>, 2>(a, nb, st); }
void launch_lines_2352_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 12, 14>, 4>(a, nb, st); }
void launch_lines_2352_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 14, 14>, 4>(a, nb, st); }
void launch_lines_2352_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 12, 14>, 2>(a, nb, st); }
void launch_lines_3840_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 15, 16>, 2>(a, nb, st); }
void launch_lines_3840_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 16, 16>, 2>(a, nb, st); }
}  // namespace dwcu
