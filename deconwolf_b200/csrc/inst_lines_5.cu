// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_6_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 2, 1>, 16>(a, nb, st); }
void launch_lines_6_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<2, 3, 1>, 16>(a, nb, st); }
void launch_lines_6_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 2, 1>, 8>(a, nb, st); }
void launch_lines_30_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 5, 1>, 16>(a, nb, st); }
void launch_lines_30_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 6, 1>, 16>(a, nb, st); }
void launch_lines_30_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 5, 1>, 8>(a, nb, st); }
void launch_lines_72_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 8, 1>, 16>(a, nb, st); }
void launch_lines_72_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 9, 1>, 16>(a, nb, st); }
void launch_lines_72_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 8, 1>, 8>(a, nb, st); }
void launch_lines_135_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 1>, 16>(a, nb, st); }
void launch_lines_135_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 15, 1>, 16>(a, nb, st); }
void launch_lines_135_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 1>, 8>(a, nb, st); }
void launch_lines_224_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 14, 1>, 16>(a, nb, st); }
void launch_lines_224_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 16, 1>, 16>(a, nb, st); }
void launch_lines_224_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 14, 1>, 8>(a, nb, st); }
void launch_lines_336_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 7>, 16>(a, nb, st); }
void launch_lines_336_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 6, 8>, 16>(a, nb, st); }
void launch_lines_336_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 7>, 8>(a, nb, st); }
void launch_lines_486_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 9>, 8>(a, nb, st); }
void launch_lines_486_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 9, 9>, 8>(a, nb, st); }
void launch_lines_486_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 9>, 4>(a, nb, st); }
void launch_lines_675_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 9>, 4>(a, nb, st); }
void launch_lines_675_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 15>, 4>(a, nb, st); }
void launch_lines_675_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 9>, 2>(a, nb, st); }
void launch_lines_900_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 9, 10>, 8>(a, nb, st); }
void launch_lines_900_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 10, 10>, 8>(a, nb, st); }
void launch_lines_900_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 9, 10>, 4>(a, nb, st); }
void launch_lines_1215_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 9>, 4>(a, nb, st); }
void launch_lines_1215_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 9, 15>, 4>(a, nb, st); }
void launch_lines_1215_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 9>, 2>(a, nb, st); }
void launch_lines_1620_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 12>, 4>(a, nb, st); }
void launch_lines_1620_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 15>, 4>(a, nb, st); }
void launch_lines_1620_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 12>, 2>(a, nb, st); }
void launch_lines_2304_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 12>, 4>(a, nb, st); }
void launch_lines_2304_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 12, 16>, 4>(a, nb, st); }
void launch_lines_2304_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 12>, 2>(a, nb, st); }
void launch_lines_3600_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 15, 15>, 2>(a, nb, st); }
void launch_lines_3600_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 15, 16>, 2>(a, nb, st); }
}  // namespace dwcu
