// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_14_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 2, 1>, 16>(a, nb, st); }
void launch_lines_14_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<2, 7, 1>, 16>(a, nb, st); }
void launch_lines_14_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 2, 1>, 8>(a, nb, st); }
void launch_lines_45_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 1>, 16>(a, nb, st); }
void launch_lines_45_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 9, 1>, 16>(a, nb, st); }
void launch_lines_45_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 1>, 8>(a, nb, st); }
void launch_lines_96_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 1>, 16>(a, nb, st); }
void launch_lines_96_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 12, 1>, 16>(a, nb, st); }
void launch_lines_96_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 1>, 8>(a, nb, st); }
void launch_lines_162_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 3, 6>, 16>(a, nb, st); }
void launch_lines_162_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 3, 9>, 16>(a, nb, st); }
void launch_lines_162_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 3, 6>, 8>(a, nb, st); }
void launch_lines_252_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 6, 6>, 16>(a, nb, st); }
void launch_lines_252_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 6, 7>, 16>(a, nb, st); }
void launch_lines_252_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 6, 6>, 8>(a, nb, st); }
void launch_lines_384_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 8>, 16>(a, nb, st); }
void launch_lines_384_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 8, 8>, 16>(a, nb, st); }
void launch_lines_384_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 8>, 8>(a, nb, st); }
void launch_lines_540_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 9>, 8>(a, nb, st); }
void launch_lines_540_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 10>, 8>(a, nb, st); }
void launch_lines_540_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 9>, 4>(a, nb, st); }
void launch_lines_750_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 10>, 4>(a, nb, st); }
void launch_lines_750_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 15>, 4>(a, nb, st); }
void launch_lines_750_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 10>, 2>(a, nb, st); }
void launch_lines_1008_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 9>, 8>(a, nb, st); }
void launch_lines_1008_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 8, 14>, 8>(a, nb, st); }
void launch_lines_1008_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 9>, 4>(a, nb, st); }
void launch_lines_1372_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 14>, 4>(a, nb, st); }
void launch_lines_1372_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 14, 14>, 4>(a, nb, st); }
void launch_lines_1372_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 14>, 2>(a, nb, st); }
void launch_lines_1890_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 14>, 4>(a, nb, st); }
void launch_lines_1890_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 15>, 4>(a, nb, st); }
void launch_lines_1890_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 14>, 2>(a, nb, st); }
void launch_lines_2700_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 15>, 4>(a, nb, st); }
void launch_lines_2700_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 15, 15>, 4>(a, nb, st); }
void launch_lines_2700_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 15>, 2>(a, nb, st); }
}  // namespace dwcu
