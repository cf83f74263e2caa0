// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_15(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 3, 1>, 16>(a, nb, st); }
void launch_lines_48(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 1>, 16>(a, nb, st); }
void launch_lines_98(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 1>, 16>(a, nb, st); }
void launch_lines_168(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 12, 1>, 16>(a, nb, st); }
void launch_lines_256(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 16, 1>, 16>(a, nb, st); }
void launch_lines_392(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 7>, 16>(a, nb, st); }
void launch_lines_560(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 8>, 8>(a, nb, st); }
void launch_lines_756(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 9>, 8>(a, nb, st); }
void launch_lines_1024(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 8>, 8>(a, nb, st); }
void launch_lines_1400(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 10>, 4>(a, nb, st); }
void launch_lines_1920(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 12>, 4>(a, nb, st); }
void launch_lines_2744(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 14, 14>, 4>(a, nb, st); }
}  // namespace dwcu
