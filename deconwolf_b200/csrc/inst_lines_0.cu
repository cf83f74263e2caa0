// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_1_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<1, 1, 1>, 16>(a, nb, st); }
void launch_lines_21_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 3, 1>, 16>(a, nb, st); }
void launch_lines_21_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 7, 1>, 16>(a, nb, st); }
void launch_lines_21_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 3, 1>, 8>(a, nb, st); }
void launch_lines_56_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 1>, 16>(a, nb, st); }
void launch_lines_56_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 8, 1>, 16>(a, nb, st); }
void launch_lines_56_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 1>, 8>(a, nb, st); }
void launch_lines_112_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 1>, 16>(a, nb, st); }
void launch_lines_112_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 14, 1>, 16>(a, nb, st); }
void launch_lines_112_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 1>, 8>(a, nb, st); }
void launch_lines_192_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 1>, 16>(a, nb, st); }
void launch_lines_192_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 16, 1>, 16>(a, nb, st); }
void launch_lines_192_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 1>, 8>(a, nb, st); }
void launch_lines_294_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 6, 7>, 16>(a, nb, st); }
void launch_lines_294_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 7, 7>, 16>(a, nb, st); }
void launch_lines_294_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 6, 7>, 8>(a, nb, st); }
void launch_lines_432_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 8>, 8>(a, nb, st); }
void launch_lines_432_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 9>, 8>(a, nb, st); }
void launch_lines_432_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 8>, 4>(a, nb, st); }
void launch_lines_600_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 10>, 8>(a, nb, st); }
void launch_lines_600_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 10, 10>, 8>(a, nb, st); }
void launch_lines_600_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 10>, 4>(a, nb, st); }
void launch_lines_810_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 9, 9>, 8>(a, nb, st); }
void launch_lines_810_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 9, 10>, 8>(a, nb, st); }
void launch_lines_810_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 9, 9>, 4>(a, nb, st); }
void launch_lines_1125_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 15>, 4>(a, nb, st); }
void launch_lines_1125_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 15, 15>, 4>(a, nb, st); }
void launch_lines_1125_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 15>, 2>(a, nb, st); }
void launch_lines_1512_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 12>, 4>(a, nb, st); }
void launch_lines_1512_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 14>, 4>(a, nb, st); }
void launch_lines_1512_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 12>, 2>(a, nb, st); }
void launch_lines_2048_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 16>, 4>(a, nb, st); }
void launch_lines_2048_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 16, 16>, 4>(a, nb, st); }
void launch_lines_2048_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 16>, 2>(a, nb, st); }
void launch_lines_3136_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 14, 14>, 2>(a, nb, st); }
void launch_lines_3136_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 14, 16>, 2>(a, nb, st); }
}  // namespace dwcu
