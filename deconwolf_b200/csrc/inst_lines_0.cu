// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<1, 1, 1>, 16>(a, nb, st); }
void launch_lines_21(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 3, 1>, 16>(a, nb, st); }
void launch_lines_56(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 1>, 16>(a, nb, st); }
void launch_lines_112(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 1>, 16>(a, nb, st); }
void launch_lines_192(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 1>, 16>(a, nb, st); }
void launch_lines_294(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 6, 7>, 16>(a, nb, st); }
void launch_lines_432(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 8>, 8>(a, nb, st); }
void launch_lines_600(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 10>, 8>(a, nb, st); }
void launch_lines_810(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 9, 9>, 8>(a, nb, st); }
void launch_lines_1125(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 15>, 4>(a, nb, st); }
void launch_lines_1512(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 9, 12>, 4>(a, nb, st); }
void launch_lines_2048(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 16>, 4>(a, nb, st); }
void launch_lines_3136(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 14, 14>, 2>(a, nb, st); }
}  // namespace dwcu
