// generated by gen_plans.py -- do not edit
#include "launch.cuh"
namespace dwcu {
void launch_lines_8(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<4, 2, 1>, 16>(a, nb, st); }
void launch_lines_35(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<7, 5, 1>, 16>(a, nb, st); }
void launch_lines_80(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 8, 1>, 16>(a, nb, st); }
void launch_lines_144(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 12, 1>, 16>(a, nb, st); }
void launch_lines_240(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 15, 1>, 16>(a, nb, st); }
void launch_lines_350(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 7>, 8>(a, nb, st); }
void launch_lines_500(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 5, 10>, 8>(a, nb, st); }
void launch_lines_700(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<10, 7, 10>, 8>(a, nb, st); }
void launch_lines_960(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 8, 10>, 8>(a, nb, st); }
void launch_lines_1280(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 8, 10>, 4>(a, nb, st); }
void launch_lines_1728(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<12, 12, 12>, 4>(a, nb, st); }
void launch_lines_2400(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 10, 15>, 4>(a, nb, st); }
void launch_lines_4096(const LinesArgs &a, int nb, cudaStream_t st) { launch_lines_t<Rad<16, 16, 16>, 2>(a, nb, st); }
}  // namespace dwcu
