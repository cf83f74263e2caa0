// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_8_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 2, 1>, 16>(a, nb, st); }
void launch_lines_8_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<2, 4, 1>, 16>(a, nb, st); }
void launch_lines_8_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 2, 1>, 8>(a, nb, st); }
void launch_lines_35_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 1>, 16>(a, nb, st); }
void launch_lines_35_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 7, 1>, 16>(a, nb, st); }
void launch_lines_35_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 1>, 8>(a, nb, st); }
void launch_lines_80_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 1>, 16>(a, nb, st); }
void launch_lines_80_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 10, 1>, 16>(a, nb, st); }
void launch_lines_80_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 1>, 8>(a, nb, st); }
void launch_lines_144_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 12, 1>, 16>(a, nb, st); }
void launch_lines_144_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 9, 1>, 16>(a, nb, st); }
void launch_lines_144_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 12, 1>, 8>(a, nb, st); }
void launch_lines_240_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 15, 1>, 16>(a, nb, st); }
void launch_lines_240_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 16, 1>, 16>(a, nb, st); }
void launch_lines_240_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 15, 1>, 8>(a, nb, st); }
void launch_lines_350_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 7>, 8>(a, nb, st); }
void launch_lines_350_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 10>, 8>(a, nb, st); }
void launch_lines_350_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 7>, 4>(a, nb, st); }
void launch_lines_500_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 10>, 8>(a, nb, st); }
void launch_lines_500_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 10, 10>, 8>(a, nb, st); }
void launch_lines_500_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 10>, 4>(a, nb, st); }
void launch_lines_700_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 10>, 8>(a, nb, st); }
void launch_lines_700_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 10, 10>, 8>(a, nb, st); }
void launch_lines_700_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 10>, 4>(a, nb, st); }
void launch_lines_960_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 10>, 8>(a, nb, st); }
void launch_lines_960_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 12>, 8>(a, nb, st); }
void launch_lines_960_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 10>, 4>(a, nb, st); }
void launch_lines_1280_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 10>, 4>(a, nb, st); }
void launch_lines_1280_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 16>, 4>(a, nb, st); }
void launch_lines_1280_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 10>, 2>(a, nb, st); }
void launch_lines_1728_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 12, 12>, 4>(a, nb, st); }
void launch_lines_1728_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 9, 12>, 4>(a, nb, st); }
void launch_lines_1728_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 12, 12>, 2>(a, nb, st); }
void launch_lines_2400_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 15>, 4>(a, nb, st); }
void launch_lines_2400_1(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 16>, 4>(a, nb, st); }
void launch_lines_2400_2(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 15>, 2>(a, nb, st); }
void launch_lines_4096_0(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 16, 16>, 2>(a, nb, st); }
}  // namespace dwcu
