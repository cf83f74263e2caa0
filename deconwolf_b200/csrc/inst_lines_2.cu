// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_3(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 1, 1>, 16>(a, nb, st); }
void launch_lines_25(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 5, 1>, 16>(a, nb, st); }
void launch_lines_63(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 7, 1>, 16>(a, nb, st); }
void launch_lines_125(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 5, 5>, 16>(a, nb, st); }
void launch_lines_200(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 5, 5>, 16>(a, nb, st); }
void launch_lines_315(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 7>, 16>(a, nb, st); }
void launch_lines_448(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 8>, 16>(a, nb, st); }
void launch_lines_640(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 8>, 8>(a, nb, st); }
void launch_lines_864(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 9>, 8>(a, nb, st); }
void launch_lines_1152(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 12>, 4>(a, nb, st); }
void launch_lines_1568(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 14>, 4>(a, nb, st); }
void launch_lines_2160(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 12>, 4>(a, nb, st); }
void launch_lines_3360(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 14, 15>, 2>(a, nb, st); }
}  // namespace dwcu
