// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_6(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<3, 2, 1>, 16>(a, nb, st); }
void launch_lines_30(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<6, 5, 1>, 16>(a, nb, st); }
void launch_lines_72(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 8, 1>, 16>(a, nb, st); }
void launch_lines_135(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 1>, 16>(a, nb, st); }
void launch_lines_224(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 14, 1>, 16>(a, nb, st); }
void launch_lines_336(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 7>, 16>(a, nb, st); }
void launch_lines_486(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 9>, 8>(a, nb, st); }
void launch_lines_675(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 9>, 4>(a, nb, st); }
void launch_lines_900(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 9, 10>, 8>(a, nb, st); }
void launch_lines_1215(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 9>, 4>(a, nb, st); }
void launch_lines_1620(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 12>, 4>(a, nb, st); }
void launch_lines_2304(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 12>, 4>(a, nb, st); }
void launch_lines_3600(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 15, 15>, 2>(a, nb, st); }
}  // namespace dwcu
