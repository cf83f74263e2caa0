// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_12_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 3, 1>, 16>(a, nb, st); }
void launch_lines_12_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 4, 1>, 16>(a, nb, st); }
void launch_lines_12_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 3, 1>, 8>(a, nb, st); }
void launch_lines_42_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 6, 1>, 16>(a, nb, st); }
void launch_lines_42_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 7, 1>, 16>(a, nb, st); }
void launch_lines_42_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 6, 1>, 8>(a, nb, st); }
void launch_lines_90_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 9, 1>, 16>(a, nb, st); }
void launch_lines_90_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 10, 1>, 16>(a, nb, st); }
void launch_lines_90_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 9, 1>, 8>(a, nb, st); }
void launch_lines_160_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 1>, 16>(a, nb, st); }
void launch_lines_160_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 16, 1>, 16>(a, nb, st); }
void launch_lines_160_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 1>, 8>(a, nb, st); }
void launch_lines_250_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 5>, 16>(a, nb, st); }
void launch_lines_250_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 5, 10>, 16>(a, nb, st); }
void launch_lines_250_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 5>, 8>(a, nb, st); }
void launch_lines_378_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 7>, 16>(a, nb, st); }
void launch_lines_378_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 6, 9>, 16>(a, nb, st); }
void launch_lines_378_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 7>, 8>(a, nb, st); }
void launch_lines_525_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 7>, 8>(a, nb, st); }
void launch_lines_525_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 15>, 8>(a, nb, st); }
void launch_lines_525_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 7>, 4>(a, nb, st); }
void launch_lines_735_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 7>, 8>(a, nb, st); }
void launch_lines_735_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 7, 15>, 8>(a, nb, st); }
void launch_lines_735_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 7, 7>, 4>(a, nb, st); }
void launch_lines_1000_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 10, 10>, 8>(a, nb, st); }
void launch_lines_1000_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 10, 10>, 4>(a, nb, st); }
void launch_lines_1350_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 10>, 4>(a, nb, st); }
void launch_lines_1350_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 9, 15>, 4>(a, nb, st); }
void launch_lines_1350_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 10>, 2>(a, nb, st); }
void launch_lines_1800_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 12>, 4>(a, nb, st); }
void launch_lines_1800_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 10, 15>, 4>(a, nb, st); }
void launch_lines_1800_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 12>, 2>(a, nb, st); }
void launch_lines_2688_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 14>, 4>(a, nb, st); }
void launch_lines_2688_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 12, 16>, 4>(a, nb, st); }
void launch_lines_2688_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 14>, 2>(a, nb, st); }
}  // namespace dwcu
