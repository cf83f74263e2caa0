// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<2, 1, 1>, 16>(a, nb, st); }
void launch_lines_24(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 4, 1>, 16>(a, nb, st); }
void launch_lines_60(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 1>, 16>(a, nb, st); }
void launch_lines_120(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 10, 1>, 16>(a, nb, st); }
void launch_lines_196(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 14, 1>, 16>(a, nb, st); }
void launch_lines_300(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 6>, 16>(a, nb, st); }
void launch_lines_441(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 7>, 16>(a, nb, st); }
void launch_lines_630(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 9>, 8>(a, nb, st); }
void launch_lines_840(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 10>, 8>(a, nb, st); }
void launch_lines_1134(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 9>, 8>(a, nb, st); }
void launch_lines_1536(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 12>, 4>(a, nb, st); }
void launch_lines_2100(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 14>, 4>(a, nb, st); }
void launch_lines_3150(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 14, 15>, 2>(a, nb, st); }
}  // namespace dwcu
