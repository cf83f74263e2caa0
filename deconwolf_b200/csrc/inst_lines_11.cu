// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_14(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 2, 1>, 16>(a, nb, st); }
void launch_lines_45(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 5, 1>, 16>(a, nb, st); }
void launch_lines_96(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 1>, 16>(a, nb, st); }
void launch_lines_162(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 3, 6>, 16>(a, nb, st); }
void launch_lines_252(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 6, 6>, 16>(a, nb, st); }
void launch_lines_384(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 8>, 16>(a, nb, st); }
void launch_lines_540(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 9>, 8>(a, nb, st); }
void launch_lines_750(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 5, 10>, 4>(a, nb, st); }
void launch_lines_1008(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 9>, 8>(a, nb, st); }
void launch_lines_1372(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 7, 14>, 4>(a, nb, st); }
void launch_lines_1890(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 14>, 4>(a, nb, st); }
void launch_lines_2700(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 12, 15>, 4>(a, nb, st); }
}  // namespace dwcu
