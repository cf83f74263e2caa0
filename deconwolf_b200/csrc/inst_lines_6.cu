// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_7(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 1, 1>, 16>(a, nb, st); }
void launch_lines_32(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 4, 1>, 16>(a, nb, st); }
void launch_lines_75(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 1>, 16>(a, nb, st); }
void launch_lines_140(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 1>, 16>(a, nb, st); }
void launch_lines_225(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 15, 1>, 16>(a, nb, st); }
void launch_lines_343(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 7, 7>, 16>(a, nb, st); }
void launch_lines_490(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 7>, 8>(a, nb, st); }
void launch_lines_686(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 7>, 8>(a, nb, st); }
void launch_lines_945(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 9>, 4>(a, nb, st); }
void launch_lines_1260(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 10>, 4>(a, nb, st); }
void launch_lines_1680(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 10, 12>, 4>(a, nb, st); }
void launch_lines_2352(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 12, 14>, 4>(a, nb, st); }
void launch_lines_3840(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 15, 16>, 2>(a, nb, st); }
}  // namespace dwcu
