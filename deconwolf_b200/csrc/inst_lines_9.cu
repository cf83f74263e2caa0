// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_10(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 2, 1>, 16>(a, nb, st); }
void launch_lines_40(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 1>, 16>(a, nb, st); }
void launch_lines_84(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 1>, 16>(a, nb, st); }
void launch_lines_150(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 1>, 16>(a, nb, st); }
void launch_lines_245(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 7>, 16>(a, nb, st); }
void launch_lines_375(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 5>, 8>(a, nb, st); }
void launch_lines_512(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 8, 8>, 16>(a, nb, st); }
void launch_lines_729(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 9, 9>, 8>(a, nb, st); }
void launch_lines_980(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 10>, 4>(a, nb, st); }
void launch_lines_1344(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 12>, 4>(a, nb, st); }
void launch_lines_1792(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 14>, 4>(a, nb, st); }
void launch_lines_2560(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 16>, 4>(a, nb, st); }
}  // namespace dwcu
