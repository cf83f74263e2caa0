// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_15_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 3, 1>, 16>(a, nb, st); }
void launch_lines_15_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 5, 1>, 16>(a, nb, st); }
void launch_lines_15_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 3, 1>, 8>(a, nb, st); }
void launch_lines_48_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 1>, 16>(a, nb, st); }
void launch_lines_48_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 8, 1>, 16>(a, nb, st); }
void launch_lines_48_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 1>, 8>(a, nb, st); }
void launch_lines_98_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 1>, 16>(a, nb, st); }
void launch_lines_98_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 14, 1>, 16>(a, nb, st); }
void launch_lines_98_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 1>, 8>(a, nb, st); }
void launch_lines_168_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 12, 1>, 16>(a, nb, st); }
void launch_lines_168_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 14, 1>, 16>(a, nb, st); }
void launch_lines_168_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 12, 1>, 8>(a, nb, st); }
void launch_lines_256_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 16, 1>, 16>(a, nb, st); }
void launch_lines_256_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 4, 8>, 16>(a, nb, st); }
void launch_lines_256_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 16, 1>, 8>(a, nb, st); }
void launch_lines_392_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 7>, 16>(a, nb, st); }
void launch_lines_392_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 7, 8>, 16>(a, nb, st); }
void launch_lines_392_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 7>, 8>(a, nb, st); }
void launch_lines_560_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 8>, 8>(a, nb, st); }
void launch_lines_560_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 10>, 8>(a, nb, st); }
void launch_lines_560_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 8>, 4>(a, nb, st); }
void launch_lines_756_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 9>, 8>(a, nb, st); }
void launch_lines_756_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 12>, 8>(a, nb, st); }
void launch_lines_756_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 9>, 4>(a, nb, st); }
void launch_lines_1024_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 8>, 8>(a, nb, st); }
void launch_lines_1024_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 8, 16>, 8>(a, nb, st); }
void launch_lines_1024_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 8>, 4>(a, nb, st); }
void launch_lines_1400_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 10>, 4>(a, nb, st); }
void launch_lines_1400_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 10, 14>, 4>(a, nb, st); }
void launch_lines_1400_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 10>, 2>(a, nb, st); }
void launch_lines_1920_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 12>, 4>(a, nb, st); }
void launch_lines_1920_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 10, 16>, 4>(a, nb, st); }
void launch_lines_1920_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 12>, 2>(a, nb, st); }
void launch_lines_2744_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 14, 14>, 4>(a, nb, st); }
void launch_lines_2744_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 14, 14>, 2>(a, nb, st); }
}  // namespace dwcu
