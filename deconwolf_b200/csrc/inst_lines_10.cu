// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_12(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 3, 1>, 16>(a, nb, st); }
void launch_lines_42(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 6, 1>, 16>(a, nb, st); }
void launch_lines_90(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 9, 1>, 16>(a, nb, st); }
void launch_lines_160(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 1>, 16>(a, nb, st); }
void launch_lines_250(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 5>, 16>(a, nb, st); }
void launch_lines_378(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 7>, 16>(a, nb, st); }
void launch_lines_525(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 7>, 8>(a, nb, st); }
void launch_lines_735(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 7>, 8>(a, nb, st); }
void launch_lines_1000(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 10, 10>, 8>(a, nb, st); }
void launch_lines_1350(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 10>, 4>(a, nb, st); }
void launch_lines_1800(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 12>, 4>(a, nb, st); }
void launch_lines_2688(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 14>, 4>(a, nb, st); }
}  // namespace dwcu
