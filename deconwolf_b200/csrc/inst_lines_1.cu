// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_2_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<2, 1, 1>, 16>(a, nb, st); }
void launch_lines_2_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<2, 1, 1>, 8>(a, nb, st); }
void launch_lines_24_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 4, 1>, 16>(a, nb, st); }
void launch_lines_24_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 6, 1>, 16>(a, nb, st); }
void launch_lines_24_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 4, 1>, 8>(a, nb, st); }
void launch_lines_60_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 1>, 16>(a, nb, st); }
void launch_lines_60_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 10, 1>, 16>(a, nb, st); }
void launch_lines_60_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 1>, 8>(a, nb, st); }
void launch_lines_120_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 10, 1>, 16>(a, nb, st); }
void launch_lines_120_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 12, 1>, 16>(a, nb, st); }
void launch_lines_120_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 10, 1>, 8>(a, nb, st); }
void launch_lines_196_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 14, 1>, 16>(a, nb, st); }
void launch_lines_196_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 4, 7>, 16>(a, nb, st); }
void launch_lines_196_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 14, 1>, 8>(a, nb, st); }
void launch_lines_300_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 6>, 16>(a, nb, st); }
void launch_lines_300_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 5, 10>, 16>(a, nb, st); }
void launch_lines_300_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 6>, 8>(a, nb, st); }
void launch_lines_441_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 7>, 16>(a, nb, st); }
void launch_lines_441_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 7, 9>, 16>(a, nb, st); }
void launch_lines_441_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 7>, 8>(a, nb, st); }
void launch_lines_630_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 9>, 8>(a, nb, st); }
void launch_lines_630_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 10>, 8>(a, nb, st); }
void launch_lines_630_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 9>, 4>(a, nb, st); }
void launch_lines_840_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 10>, 8>(a, nb, st); }
void launch_lines_840_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 12>, 8>(a, nb, st); }
void launch_lines_840_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 10>, 4>(a, nb, st); }
void launch_lines_1134_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 9>, 8>(a, nb, st); }
void launch_lines_1134_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 9, 14>, 8>(a, nb, st); }
void launch_lines_1134_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 9>, 4>(a, nb, st); }
void launch_lines_1536_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 12>, 4>(a, nb, st); }
void launch_lines_1536_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 16>, 4>(a, nb, st); }
void launch_lines_1536_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 12>, 2>(a, nb, st); }
void launch_lines_2100_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 14>, 4>(a, nb, st); }
void launch_lines_2100_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 15>, 4>(a, nb, st); }
void launch_lines_2100_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 14>, 2>(a, nb, st); }
void launch_lines_3150_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 14, 15>, 2>(a, nb, st); }
void launch_lines_3150_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 15, 15>, 2>(a, nb, st); }
}  // namespace dwcu
