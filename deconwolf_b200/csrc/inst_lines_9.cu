// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_10_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 2, 1>, 16>(a, nb, st); }
void launch_lines_10_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<2, 5, 1>, 16>(a, nb, st); }
void launch_lines_10_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 2, 1>, 8>(a, nb, st); }
void launch_lines_40_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 1>, 16>(a, nb, st); }
void launch_lines_40_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 8, 1>, 16>(a, nb, st); }
void launch_lines_40_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 1>, 8>(a, nb, st); }
void launch_lines_84_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 1>, 16>(a, nb, st); }
void launch_lines_84_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 12, 1>, 16>(a, nb, st); }
void launch_lines_84_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 1>, 8>(a, nb, st); }
void launch_lines_150_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 1>, 16>(a, nb, st); }
void launch_lines_150_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 15, 1>, 16>(a, nb, st); }
void launch_lines_150_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 1>, 8>(a, nb, st); }
void launch_lines_245_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 7>, 16>(a, nb, st); }
void launch_lines_245_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 7, 7>, 16>(a, nb, st); }
void launch_lines_245_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 7>, 8>(a, nb, st); }
void launch_lines_375_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 5>, 8>(a, nb, st); }
void launch_lines_375_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 5, 15>, 8>(a, nb, st); }
void launch_lines_375_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 5>, 4>(a, nb, st); }
void launch_lines_512_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 8, 8>, 16>(a, nb, st); }
void launch_lines_512_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 4, 8>, 8>(a, nb, st); }
void launch_lines_512_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 8, 8>, 8>(a, nb, st); }
void launch_lines_729_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 9, 9>, 8>(a, nb, st); }
void launch_lines_729_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 9, 9>, 4>(a, nb, st); }
void launch_lines_980_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 10>, 4>(a, nb, st); }
void launch_lines_980_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 14>, 4>(a, nb, st); }
void launch_lines_980_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 10>, 2>(a, nb, st); }
void launch_lines_1344_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 12>, 4>(a, nb, st); }
void launch_lines_1344_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 14>, 4>(a, nb, st); }
void launch_lines_1344_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 12>, 2>(a, nb, st); }
void launch_lines_1792_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 14>, 4>(a, nb, st); }
void launch_lines_1792_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 16>, 4>(a, nb, st); }
void launch_lines_1792_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 14>, 2>(a, nb, st); }
void launch_lines_2560_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 16>, 4>(a, nb, st); }
void launch_lines_2560_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 16, 16>, 4>(a, nb, st); }
void launch_lines_2560_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 16>, 2>(a, nb, st); }
}  // namespace dwcu
