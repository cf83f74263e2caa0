// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_4_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<2, 2, 1>, 16>(a, nb, st); }
void launch_lines_4_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 1, 1>, 16>(a, nb, st); }
void launch_lines_4_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<2, 2, 1>, 8>(a, nb, st); }
void launch_lines_27_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 3, 1>, 16>(a, nb, st); }
void launch_lines_27_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 9, 1>, 16>(a, nb, st); }
void launch_lines_27_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 3, 1>, 8>(a, nb, st); }
void launch_lines_64_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 8, 1>, 16>(a, nb, st); }
void launch_lines_64_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 4, 1>, 16>(a, nb, st); }
void launch_lines_64_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 8, 1>, 8>(a, nb, st); }
void launch_lines_126_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 1>, 16>(a, nb, st); }
void launch_lines_126_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 14, 1>, 16>(a, nb, st); }
void launch_lines_126_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 1>, 8>(a, nb, st); }
void launch_lines_210_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 14, 1>, 16>(a, nb, st); }
void launch_lines_210_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 15, 1>, 16>(a, nb, st); }
void launch_lines_210_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 14, 1>, 8>(a, nb, st); }
void launch_lines_320_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 8>, 16>(a, nb, st); }
void launch_lines_320_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 8, 8>, 16>(a, nb, st); }
void launch_lines_320_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 8>, 8>(a, nb, st); }
void launch_lines_450_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 9>, 8>(a, nb, st); }
void launch_lines_450_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 10>, 8>(a, nb, st); }
void launch_lines_450_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 9>, 4>(a, nb, st); }
void launch_lines_648_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 8, 9>, 8>(a, nb, st); }
void launch_lines_648_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 9, 9>, 8>(a, nb, st); }
void launch_lines_648_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 8, 9>, 4>(a, nb, st); }
void launch_lines_882_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 9>, 8>(a, nb, st); }
void launch_lines_882_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 14>, 8>(a, nb, st); }
void launch_lines_882_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 9>, 4>(a, nb, st); }
void launch_lines_1176_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 12>, 4>(a, nb, st); }
void launch_lines_1176_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 14>, 4>(a, nb, st); }
void launch_lines_1176_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 12>, 2>(a, nb, st); }
void launch_lines_1575_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 15>, 4>(a, nb, st); }
void launch_lines_1575_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 15, 15>, 4>(a, nb, st); }
void launch_lines_1575_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 15>, 2>(a, nb, st); }
void launch_lines_2240_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 14>, 4>(a, nb, st); }
void launch_lines_2240_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 16>, 4>(a, nb, st); }
void launch_lines_2240_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 14>, 2>(a, nb, st); }
void launch_lines_3375_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 15, 15>, 2>(a, nb, st); }
}  // namespace dwcu
