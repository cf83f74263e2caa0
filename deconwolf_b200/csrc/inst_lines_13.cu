// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_16_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 4, 1>, 16>(a, nb, st); }
void launch_lines_16_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 2, 1>, 16>(a, nb, st); }
void launch_lines_16_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 4, 1>, 8>(a, nb, st); }
void launch_lines_49_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 7, 1>, 16>(a, nb, st); }
void launch_lines_49_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 7, 1>, 8>(a, nb, st); }
void launch_lines_100_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 10, 1>, 16>(a, nb, st); }
void launch_lines_100_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 4, 5>, 16>(a, nb, st); }
void launch_lines_100_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 10, 1>, 8>(a, nb, st); }
void launch_lines_175_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 5>, 16>(a, nb, st); }
void launch_lines_175_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 5, 7>, 16>(a, nb, st); }
void launch_lines_175_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 5>, 8>(a, nb, st); }
void launch_lines_270_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 6>, 16>(a, nb, st); }
void launch_lines_270_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 5, 9>, 16>(a, nb, st); }
void launch_lines_270_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 6>, 8>(a, nb, st); }
void launch_lines_400_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 8>, 8>(a, nb, st); }
void launch_lines_400_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 10>, 8>(a, nb, st); }
void launch_lines_400_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 8>, 4>(a, nb, st); }
void launch_lines_567_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 9>, 8>(a, nb, st); }
void launch_lines_567_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 9, 9>, 8>(a, nb, st); }
void launch_lines_567_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 9>, 4>(a, nb, st); }
void launch_lines_768_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 8>, 8>(a, nb, st); }
void launch_lines_768_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 8, 12>, 8>(a, nb, st); }
void launch_lines_768_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 8>, 4>(a, nb, st); }
void launch_lines_1050_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 10>, 4>(a, nb, st); }
void launch_lines_1050_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 15>, 4>(a, nb, st); }
void launch_lines_1050_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 10>, 2>(a, nb, st); }
void launch_lines_1440_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 10, 12>, 4>(a, nb, st); }
void launch_lines_1440_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 12, 12>, 4>(a, nb, st); }
void launch_lines_1440_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 10, 12>, 2>(a, nb, st); }
void launch_lines_1960_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 14>, 4>(a, nb, st); }
void launch_lines_1960_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 14, 14>, 4>(a, nb, st); }
void launch_lines_1960_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 14>, 2>(a, nb, st); }
void launch_lines_2880_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 15>, 4>(a, nb, st); }
void launch_lines_2880_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 16>, 4>(a, nb, st); }
void launch_lines_2880_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 15>, 2>(a, nb, st); }
}  // namespace dwcu
