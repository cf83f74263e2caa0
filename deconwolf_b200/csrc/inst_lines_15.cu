// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_20(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<5, 4, 1>, 16>(a, nb, st); }
void launch_lines_54(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 6, 1>, 16>(a, nb, st); }
void launch_lines_108(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 9, 1>, 16>(a, nb, st); }
void launch_lines_189(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<9, 3, 7>, 16>(a, nb, st); }
void launch_lines_288(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<8, 6, 6>, 16>(a, nb, st); }
void launch_lines_420(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 6, 7>, 8>(a, nb, st); }
void launch_lines_588(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 7, 7>, 8>(a, nb, st); }
void launch_lines_800(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 10>, 8>(a, nb, st); }
void launch_lines_1120(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<14, 8, 10>, 4>(a, nb, st); }
void launch_lines_1500(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 10, 10>, 4>(a, nb, st); }
void launch_lines_2025(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<15, 9, 15>, 4>(a, nb, st); }
void launch_lines_3072(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 12, 16>, 2>(a, nb, st); }
}  // namespace dwcu
