// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_4(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<2, 2, 1>, 16>(a, nb, st); }
void launch_lines_27(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 3, 1>, 16>(a, nb, st); }
void launch_lines_64(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 8, 1>, 16>(a, nb, st); }
void launch_lines_126(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 1>, 16>(a, nb, st); }
void launch_lines_210(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 14, 1>, 16>(a, nb, st); }
void launch_lines_320(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 8>, 16>(a, nb, st); }
void launch_lines_450(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 9>, 8>(a, nb, st); }
void launch_lines_648(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 8, 9>, 8>(a, nb, st); }
void launch_lines_882(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 9>, 8>(a, nb, st); }
void launch_lines_1176(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 12>, 4>(a, nb, st); }
void launch_lines_1575(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 15>, 4>(a, nb, st); }
void launch_lines_2240(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 14>, 4>(a, nb, st); }
void launch_lines_3375(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 15, 15>, 2>(a, nb, st); }
}  // namespace dwcu
