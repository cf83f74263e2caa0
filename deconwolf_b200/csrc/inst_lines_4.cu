// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_5(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 1, 1>, 16>(a, nb, st); }
void launch_lines_28(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 4, 1>, 16>(a, nb, st); }
void launch_lines_70(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 1>, 16>(a, nb, st); }
void launch_lines_128(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 1>, 16>(a, nb, st); }
void launch_lines_216(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 6, 6>, 16>(a, nb, st); }
void launch_lines_324(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 6>, 16>(a, nb, st); }
void launch_lines_480(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 8>, 8>(a, nb, st); }
void launch_lines_672(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 8>, 8>(a, nb, st); }
void launch_lines_896(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 8>, 8>(a, nb, st); }
void launch_lines_1200(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 10, 10>, 8>(a, nb, st); }
void launch_lines_1600(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 10>, 4>(a, nb, st); }
void launch_lines_2250(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 15>, 4>(a, nb, st); }
void launch_lines_3584(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 14, 16>, 2>(a, nb, st); }
}  // namespace dwcu
