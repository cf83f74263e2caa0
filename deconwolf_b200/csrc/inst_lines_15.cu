// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_20_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 4, 1>, 16>(a, nb, st); }
void launch_lines_20_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 5, 1>, 16>(a, nb, st); }
void launch_lines_20_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 4, 1>, 8>(a, nb, st); }
void launch_lines_54_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 1>, 16>(a, nb, st); }
void launch_lines_54_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 9, 1>, 16>(a, nb, st); }
void launch_lines_54_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 1>, 8>(a, nb, st); }
void launch_lines_108_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 1>, 16>(a, nb, st); }
void launch_lines_108_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 12, 1>, 16>(a, nb, st); }
void launch_lines_108_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 1>, 8>(a, nb, st); }
void launch_lines_189_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 3, 7>, 16>(a, nb, st); }
void launch_lines_189_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 3, 9>, 16>(a, nb, st); }
void launch_lines_189_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 3, 7>, 8>(a, nb, st); }
void launch_lines_288_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 6>, 16>(a, nb, st); }
void launch_lines_288_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 6, 8>, 16>(a, nb, st); }
void launch_lines_288_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 6>, 8>(a, nb, st); }
void launch_lines_420_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 7>, 8>(a, nb, st); }
void launch_lines_420_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 6, 10>, 8>(a, nb, st); }
void launch_lines_420_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 7>, 4>(a, nb, st); }
void launch_lines_588_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 7>, 8>(a, nb, st); }
void launch_lines_588_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 7, 12>, 8>(a, nb, st); }
void launch_lines_588_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 7>, 4>(a, nb, st); }
void launch_lines_800_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 10>, 8>(a, nb, st); }
void launch_lines_800_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 10, 10>, 8>(a, nb, st); }
void launch_lines_800_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 10>, 4>(a, nb, st); }
void launch_lines_1120_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 10>, 4>(a, nb, st); }
void launch_lines_1120_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 14>, 4>(a, nb, st); }
void launch_lines_1120_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 10>, 2>(a, nb, st); }
void launch_lines_1500_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 10>, 4>(a, nb, st); }
void launch_lines_1500_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 10, 15>, 4>(a, nb, st); }
void launch_lines_1500_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 10>, 2>(a, nb, st); }
void launch_lines_2025_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 15>, 4>(a, nb, st); }
void launch_lines_2025_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 15, 15>, 4>(a, nb, st); }
void launch_lines_2025_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 15>, 2>(a, nb, st); }
void launch_lines_3072_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 16>, 2>(a, nb, st); }
void launch_lines_3072_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 16, 16>, 2>(a, nb, st); }
}  // namespace dwcu
