// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_5_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 1, 1>, 16>(a, nb, st); }
void launch_lines_5_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 1, 1>, 8>(a, nb, st); }
void launch_lines_28_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 4, 1>, 16>(a, nb, st); }
void launch_lines_28_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 7, 1>, 16>(a, nb, st); }
void launch_lines_28_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 4, 1>, 8>(a, nb, st); }
void launch_lines_70_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 1>, 16>(a, nb, st); }
void launch_lines_70_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 10, 1>, 16>(a, nb, st); }
void launch_lines_70_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 1>, 8>(a, nb, st); }
void launch_lines_128_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 1>, 16>(a, nb, st); }
void launch_lines_128_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 16, 1>, 16>(a, nb, st); }
void launch_lines_128_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 1>, 8>(a, nb, st); }
void launch_lines_216_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 6, 6>, 16>(a, nb, st); }
void launch_lines_216_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 4, 6>, 16>(a, nb, st); }
void launch_lines_216_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 6, 6>, 8>(a, nb, st); }
void launch_lines_324_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 6>, 16>(a, nb, st); }
void launch_lines_324_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 6, 9>, 16>(a, nb, st); }
void launch_lines_324_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 6>, 8>(a, nb, st); }
void launch_lines_480_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 8>, 8>(a, nb, st); }
void launch_lines_480_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 10>, 8>(a, nb, st); }
void launch_lines_480_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 8>, 4>(a, nb, st); }
void launch_lines_672_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 8>, 8>(a, nb, st); }
void launch_lines_672_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 7, 12>, 8>(a, nb, st); }
void launch_lines_672_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 8>, 4>(a, nb, st); }
void launch_lines_896_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 8>, 8>(a, nb, st); }
void launch_lines_896_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 8, 14>, 8>(a, nb, st); }
void launch_lines_896_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 8>, 4>(a, nb, st); }
void launch_lines_1200_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 10, 10>, 8>(a, nb, st); }
void launch_lines_1200_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 10, 12>, 8>(a, nb, st); }
void launch_lines_1200_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 10, 10>, 4>(a, nb, st); }
void launch_lines_1600_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 10>, 4>(a, nb, st); }
void launch_lines_1600_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 10, 16>, 4>(a, nb, st); }
void launch_lines_1600_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 10>, 2>(a, nb, st); }
void launch_lines_2250_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 15>, 4>(a, nb, st); }
void launch_lines_2250_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 15, 15>, 4>(a, nb, st); }
void launch_lines_2250_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 15>, 2>(a, nb, st); }
void launch_lines_3584_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 14, 16>, 2>(a, nb, st); }
void launch_lines_3584_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 16, 16>, 2>(a, nb, st); }
}  // namespace dwcu
