// generated by gen_plans.py -- do not edit
#pragma once
#include "passes.cuh"
namespace dwcu {
// one entry per autotuning candidate of a length, candidates of a length in
// order (cand 0: the generator's heuristic choice)
struct LinesPlan { int n, cand, ra, rb, rc, T, threads; size_t smem; void (*launch)(const LinesArgs &, int, cudaStream_t); };
struct XPlan { int n, cand, ra, rb, rc, R, threads; size_t smem; void (*launch)(const XArgs &, cudaStream_t); };
struct YPlan { int n, cand, ra, rb, rc, threads; size_t smem; void (*launch)(const YArgs &, cudaStream_t); };
void launch_lines_1_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_3_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_3_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_4_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_4_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_4_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_5_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_5_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_6_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_6_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_6_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_7_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_7_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_8_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_8_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_8_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_9_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_9_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_9_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_10_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_10_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_10_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_12_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_12_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_12_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_14_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_14_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_14_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_15_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_15_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_15_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_16_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_16_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_16_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_18_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_18_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_18_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_20_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_20_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_20_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_21_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_21_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_21_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_24_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_24_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_24_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_25_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_25_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_27_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_27_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_27_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_28_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_28_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_28_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_30_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_30_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_30_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_32_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_32_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_32_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_35_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_35_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_35_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_36_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_36_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_36_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_40_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_40_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_40_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_42_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_42_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_42_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_45_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_45_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_45_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_48_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_48_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_48_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_49_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_49_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_50_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_50_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_50_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_54_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_54_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_54_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_56_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_56_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_56_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_60_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_60_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_60_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_63_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_63_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_63_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_64_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_64_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_64_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_70_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_70_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_70_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_72_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_72_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_72_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_75_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_75_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_75_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_80_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_80_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_80_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_81_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_81_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_81_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_84_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_84_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_84_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_90_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_90_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_90_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_96_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_96_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_96_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_98_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_98_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_98_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_100_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_100_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_100_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_105_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_105_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_105_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_108_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_108_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_108_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_112_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_112_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_112_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_120_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_120_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_120_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_125_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_125_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_126_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_126_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_126_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_128_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_128_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_128_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_135_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_135_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_135_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_140_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_140_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_140_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_144_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_144_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_144_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_147_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_147_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_147_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_150_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_150_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_150_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_160_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_160_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_160_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_162_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_162_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_162_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_168_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_168_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_168_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_175_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_175_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_175_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_180_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_180_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_180_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_189_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_189_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_189_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_192_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_192_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_192_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_196_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_196_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_196_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_200_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_200_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_200_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_210_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_210_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_210_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_216_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_216_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_216_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_224_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_224_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_224_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_225_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_225_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_225_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_240_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_240_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_240_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_243_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_243_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_243_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_245_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_245_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_245_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_250_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_250_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_250_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_252_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_252_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_252_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_256_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_256_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_256_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_270_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_270_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_270_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_280_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_280_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_280_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_288_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_288_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_288_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_294_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_294_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_294_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_300_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_300_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_300_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_315_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_315_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_315_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_320_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_320_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_320_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_324_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_324_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_324_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_336_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_336_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_336_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_343_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_343_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_350_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_350_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_350_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_360_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_360_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_360_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_375_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_375_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_375_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_378_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_378_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_378_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_384_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_384_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_384_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_392_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_392_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_392_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_400_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_400_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_400_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_405_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_405_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_405_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_420_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_420_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_420_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_432_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_432_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_432_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_441_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_441_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_441_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_448_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_448_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_448_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_450_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_450_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_450_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_480_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_480_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_480_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_486_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_486_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_486_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_490_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_490_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_490_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_500_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_500_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_500_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_504_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_504_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_504_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_512_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_512_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_512_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_525_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_525_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_525_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_540_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_540_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_540_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_560_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_560_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_560_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_567_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_567_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_567_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_576_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_576_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_576_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_588_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_588_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_588_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_600_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_600_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_600_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_630_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_630_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_630_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_640_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_640_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_640_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_648_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_648_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_648_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_672_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_672_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_672_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_675_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_675_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_675_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_686_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_686_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_686_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_700_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_700_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_700_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_720_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_720_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_720_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_729_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_729_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_735_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_735_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_735_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_750_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_750_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_750_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_756_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_756_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_756_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_768_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_768_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_768_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_784_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_784_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_784_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_800_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_800_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_800_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_810_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_810_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_810_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_840_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_840_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_840_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_864_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_864_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_864_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_882_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_882_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_882_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_896_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_896_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_896_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_900_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_900_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_900_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_945_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_945_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_945_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_960_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_960_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_960_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_972_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_972_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_972_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_980_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_980_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_980_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1000_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1000_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1008_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1008_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1008_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1024_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1024_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1024_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1050_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1050_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1050_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1080_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1080_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1080_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1120_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1120_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1120_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1125_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1125_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1125_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1134_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1134_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1134_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1152_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1152_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1152_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1176_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1176_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1176_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1200_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1200_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1200_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1215_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1215_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1215_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1260_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1260_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1260_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1280_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1280_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1280_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1296_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1296_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1296_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1344_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1344_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1344_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1350_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1350_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1350_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1372_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1372_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1372_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1400_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1400_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1400_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1440_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1440_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1440_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1470_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1470_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1470_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1500_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1500_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1500_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1512_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1512_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1512_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1536_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1536_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1536_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1568_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1568_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1568_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1575_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1575_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1575_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1600_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1600_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1600_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1620_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1620_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1620_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1680_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1680_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1680_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1728_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1728_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1728_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1764_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1764_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1764_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1792_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1792_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1792_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1800_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1800_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1800_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1890_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1890_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1890_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1920_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1920_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1920_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_1960_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_1960_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_1960_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2016_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2016_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2016_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2025_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2025_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2025_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2048_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2048_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2048_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2100_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2100_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2100_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2160_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2160_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2160_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2240_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2240_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2240_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2250_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2250_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2250_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2304_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2304_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2304_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2352_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2352_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2352_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2400_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2400_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2400_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2520_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2520_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2520_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2560_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2560_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2560_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2688_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2688_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2688_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2700_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2700_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2700_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2744_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2744_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2880_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2880_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2880_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_2940_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_2940_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2940_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_3072_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_3072_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_3136_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_3136_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_3150_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_3150_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_3360_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_3360_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_3375_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_3584_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_3584_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_3600_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_3600_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_3840_0(const LinesArgs &, int, cudaStream_t);
void launch_lines_3840_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_4096_0(const LinesArgs &, int, cudaStream_t);
void launch_x_2_0(const XArgs &, cudaStream_t);
void launch_x_3_0(const XArgs &, cudaStream_t);
void launch_x_4_0(const XArgs &, cudaStream_t);
void launch_x_5_0(const XArgs &, cudaStream_t);
void launch_x_6_0(const XArgs &, cudaStream_t);
void launch_x_7_0(const XArgs &, cudaStream_t);
void launch_x_8_0(const XArgs &, cudaStream_t);
void launch_x_9_0(const XArgs &, cudaStream_t);
void launch_x_10_0(const XArgs &, cudaStream_t);
void launch_x_12_0(const XArgs &, cudaStream_t);
void launch_x_14_0(const XArgs &, cudaStream_t);
void launch_x_15_0(const XArgs &, cudaStream_t);
void launch_x_16_0(const XArgs &, cudaStream_t);
void launch_x_18_0(const XArgs &, cudaStream_t);
void launch_x_20_0(const XArgs &, cudaStream_t);
void launch_x_21_0(const XArgs &, cudaStream_t);
void launch_x_24_0(const XArgs &, cudaStream_t);
void launch_x_25_0(const XArgs &, cudaStream_t);
void launch_x_27_0(const XArgs &, cudaStream_t);
void launch_x_28_0(const XArgs &, cudaStream_t);
void launch_x_30_0(const XArgs &, cudaStream_t);
void launch_x_32_0(const XArgs &, cudaStream_t);
void launch_x_35_0(const XArgs &, cudaStream_t);
void launch_x_36_0(const XArgs &, cudaStream_t);
void launch_x_40_0(const XArgs &, cudaStream_t);
void launch_x_42_0(const XArgs &, cudaStream_t);
void launch_x_45_0(const XArgs &, cudaStream_t);
void launch_x_48_0(const XArgs &, cudaStream_t);
void launch_x_49_0(const XArgs &, cudaStream_t);
void launch_x_50_0(const XArgs &, cudaStream_t);
void launch_x_54_0(const XArgs &, cudaStream_t);
void launch_x_56_0(const XArgs &, cudaStream_t);
void launch_x_60_0(const XArgs &, cudaStream_t);
void launch_x_63_0(const XArgs &, cudaStream_t);
void launch_x_64_0(const XArgs &, cudaStream_t);
void launch_x_70_0(const XArgs &, cudaStream_t);
void launch_x_72_0(const XArgs &, cudaStream_t);
void launch_x_75_0(const XArgs &, cudaStream_t);
void launch_x_80_0(const XArgs &, cudaStream_t);
void launch_x_81_0(const XArgs &, cudaStream_t);
void launch_x_84_0(const XArgs &, cudaStream_t);
void launch_x_90_0(const XArgs &, cudaStream_t);
void launch_x_96_0(const XArgs &, cudaStream_t);
void launch_x_96_1(const XArgs &, cudaStream_t);
void launch_x_98_0(const XArgs &, cudaStream_t);
void launch_x_98_1(const XArgs &, cudaStream_t);
void launch_x_100_0(const XArgs &, cudaStream_t);
void launch_x_105_0(const XArgs &, cudaStream_t);
void launch_x_105_1(const XArgs &, cudaStream_t);
void launch_x_108_0(const XArgs &, cudaStream_t);
void launch_x_108_1(const XArgs &, cudaStream_t);
void launch_x_112_0(const XArgs &, cudaStream_t);
void launch_x_112_1(const XArgs &, cudaStream_t);
void launch_x_120_0(const XArgs &, cudaStream_t);
void launch_x_120_1(const XArgs &, cudaStream_t);
void launch_x_125_0(const XArgs &, cudaStream_t);
void launch_x_126_0(const XArgs &, cudaStream_t);
void launch_x_126_1(const XArgs &, cudaStream_t);
void launch_x_128_0(const XArgs &, cudaStream_t);
void launch_x_128_1(const XArgs &, cudaStream_t);
void launch_x_135_0(const XArgs &, cudaStream_t);
void launch_x_135_1(const XArgs &, cudaStream_t);
void launch_x_140_0(const XArgs &, cudaStream_t);
void launch_x_140_1(const XArgs &, cudaStream_t);
void launch_x_144_0(const XArgs &, cudaStream_t);
void launch_x_147_0(const XArgs &, cudaStream_t);
void launch_x_147_1(const XArgs &, cudaStream_t);
void launch_x_150_0(const XArgs &, cudaStream_t);
void launch_x_150_1(const XArgs &, cudaStream_t);
void launch_x_160_0(const XArgs &, cudaStream_t);
void launch_x_160_1(const XArgs &, cudaStream_t);
void launch_x_162_0(const XArgs &, cudaStream_t);
void launch_x_162_1(const XArgs &, cudaStream_t);
void launch_x_168_0(const XArgs &, cudaStream_t);
void launch_x_168_1(const XArgs &, cudaStream_t);
void launch_x_175_0(const XArgs &, cudaStream_t);
void launch_x_175_1(const XArgs &, cudaStream_t);
void launch_x_180_0(const XArgs &, cudaStream_t);
void launch_x_180_1(const XArgs &, cudaStream_t);
void launch_x_189_0(const XArgs &, cudaStream_t);
void launch_x_189_1(const XArgs &, cudaStream_t);
void launch_x_192_0(const XArgs &, cudaStream_t);
void launch_x_192_1(const XArgs &, cudaStream_t);
void launch_x_196_0(const XArgs &, cudaStream_t);
void launch_x_200_0(const XArgs &, cudaStream_t);
void launch_x_200_1(const XArgs &, cudaStream_t);
void launch_x_210_0(const XArgs &, cudaStream_t);
void launch_x_210_1(const XArgs &, cudaStream_t);
void launch_x_216_0(const XArgs &, cudaStream_t);
void launch_x_216_1(const XArgs &, cudaStream_t);
void launch_x_224_0(const XArgs &, cudaStream_t);
void launch_x_224_1(const XArgs &, cudaStream_t);
void launch_x_225_0(const XArgs &, cudaStream_t);
void launch_x_240_0(const XArgs &, cudaStream_t);
void launch_x_240_1(const XArgs &, cudaStream_t);
void launch_x_243_0(const XArgs &, cudaStream_t);
void launch_x_243_1(const XArgs &, cudaStream_t);
void launch_x_245_0(const XArgs &, cudaStream_t);
void launch_x_245_1(const XArgs &, cudaStream_t);
void launch_x_250_0(const XArgs &, cudaStream_t);
void launch_x_250_1(const XArgs &, cudaStream_t);
void launch_x_252_0(const XArgs &, cudaStream_t);
void launch_x_252_1(const XArgs &, cudaStream_t);
void launch_x_256_0(const XArgs &, cudaStream_t);
void launch_x_270_0(const XArgs &, cudaStream_t);
void launch_x_270_1(const XArgs &, cudaStream_t);
void launch_x_280_0(const XArgs &, cudaStream_t);
void launch_x_280_1(const XArgs &, cudaStream_t);
void launch_x_288_0(const XArgs &, cudaStream_t);
void launch_x_288_1(const XArgs &, cudaStream_t);
void launch_x_294_0(const XArgs &, cudaStream_t);
void launch_x_294_1(const XArgs &, cudaStream_t);
void launch_x_300_0(const XArgs &, cudaStream_t);
void launch_x_300_1(const XArgs &, cudaStream_t);
void launch_x_315_0(const XArgs &, cudaStream_t);
void launch_x_315_1(const XArgs &, cudaStream_t);
void launch_x_320_0(const XArgs &, cudaStream_t);
void launch_x_320_1(const XArgs &, cudaStream_t);
void launch_x_324_0(const XArgs &, cudaStream_t);
void launch_x_324_1(const XArgs &, cudaStream_t);
void launch_x_336_0(const XArgs &, cudaStream_t);
void launch_x_336_1(const XArgs &, cudaStream_t);
void launch_x_343_0(const XArgs &, cudaStream_t);
void launch_x_350_0(const XArgs &, cudaStream_t);
void launch_x_350_1(const XArgs &, cudaStream_t);
void launch_x_360_0(const XArgs &, cudaStream_t);
void launch_x_360_1(const XArgs &, cudaStream_t);
void launch_x_375_0(const XArgs &, cudaStream_t);
void launch_x_375_1(const XArgs &, cudaStream_t);
void launch_x_378_0(const XArgs &, cudaStream_t);
void launch_x_378_1(const XArgs &, cudaStream_t);
void launch_x_384_0(const XArgs &, cudaStream_t);
void launch_x_384_1(const XArgs &, cudaStream_t);
void launch_x_392_0(const XArgs &, cudaStream_t);
void launch_x_392_1(const XArgs &, cudaStream_t);
void launch_x_400_0(const XArgs &, cudaStream_t);
void launch_x_400_1(const XArgs &, cudaStream_t);
void launch_x_405_0(const XArgs &, cudaStream_t);
void launch_x_405_1(const XArgs &, cudaStream_t);
void launch_x_420_0(const XArgs &, cudaStream_t);
void launch_x_420_1(const XArgs &, cudaStream_t);
void launch_x_432_0(const XArgs &, cudaStream_t);
void launch_x_432_1(const XArgs &, cudaStream_t);
void launch_x_441_0(const XArgs &, cudaStream_t);
void launch_x_441_1(const XArgs &, cudaStream_t);
void launch_x_448_0(const XArgs &, cudaStream_t);
void launch_x_448_1(const XArgs &, cudaStream_t);
void launch_x_450_0(const XArgs &, cudaStream_t);
void launch_x_450_1(const XArgs &, cudaStream_t);
void launch_x_480_0(const XArgs &, cudaStream_t);
void launch_x_480_1(const XArgs &, cudaStream_t);
void launch_x_486_0(const XArgs &, cudaStream_t);
void launch_x_486_1(const XArgs &, cudaStream_t);
void launch_x_490_0(const XArgs &, cudaStream_t);
void launch_x_490_1(const XArgs &, cudaStream_t);
void launch_x_500_0(const XArgs &, cudaStream_t);
void launch_x_500_1(const XArgs &, cudaStream_t);
void launch_x_504_0(const XArgs &, cudaStream_t);
void launch_x_504_1(const XArgs &, cudaStream_t);
void launch_x_512_0(const XArgs &, cudaStream_t);
void launch_x_512_1(const XArgs &, cudaStream_t);
void launch_x_525_0(const XArgs &, cudaStream_t);
void launch_x_525_1(const XArgs &, cudaStream_t);
void launch_x_540_0(const XArgs &, cudaStream_t);
void launch_x_540_1(const XArgs &, cudaStream_t);
void launch_x_560_0(const XArgs &, cudaStream_t);
void launch_x_560_1(const XArgs &, cudaStream_t);
void launch_x_567_0(const XArgs &, cudaStream_t);
void launch_x_567_1(const XArgs &, cudaStream_t);
void launch_x_576_0(const XArgs &, cudaStream_t);
void launch_x_576_1(const XArgs &, cudaStream_t);
void launch_x_588_0(const XArgs &, cudaStream_t);
void launch_x_588_1(const XArgs &, cudaStream_t);
void launch_x_600_0(const XArgs &, cudaStream_t);
void launch_x_600_1(const XArgs &, cudaStream_t);
void launch_x_630_0(const XArgs &, cudaStream_t);
void launch_x_630_1(const XArgs &, cudaStream_t);
void launch_x_640_0(const XArgs &, cudaStream_t);
void launch_x_640_1(const XArgs &, cudaStream_t);
void launch_x_648_0(const XArgs &, cudaStream_t);
void launch_x_648_1(const XArgs &, cudaStream_t);
void launch_x_672_0(const XArgs &, cudaStream_t);
void launch_x_672_1(const XArgs &, cudaStream_t);
void launch_x_675_0(const XArgs &, cudaStream_t);
void launch_x_675_1(const XArgs &, cudaStream_t);
void launch_x_686_0(const XArgs &, cudaStream_t);
void launch_x_686_1(const XArgs &, cudaStream_t);
void launch_x_700_0(const XArgs &, cudaStream_t);
void launch_x_700_1(const XArgs &, cudaStream_t);
void launch_x_720_0(const XArgs &, cudaStream_t);
void launch_x_720_1(const XArgs &, cudaStream_t);
void launch_x_729_0(const XArgs &, cudaStream_t);
void launch_x_735_0(const XArgs &, cudaStream_t);
void launch_x_735_1(const XArgs &, cudaStream_t);
void launch_x_750_0(const XArgs &, cudaStream_t);
void launch_x_750_1(const XArgs &, cudaStream_t);
void launch_x_756_0(const XArgs &, cudaStream_t);
void launch_x_756_1(const XArgs &, cudaStream_t);
void launch_x_768_0(const XArgs &, cudaStream_t);
void launch_x_768_1(const XArgs &, cudaStream_t);
void launch_x_784_0(const XArgs &, cudaStream_t);
void launch_x_784_1(const XArgs &, cudaStream_t);
void launch_x_800_0(const XArgs &, cudaStream_t);
void launch_x_800_1(const XArgs &, cudaStream_t);
void launch_x_810_0(const XArgs &, cudaStream_t);
void launch_x_810_1(const XArgs &, cudaStream_t);
void launch_x_840_0(const XArgs &, cudaStream_t);
void launch_x_840_1(const XArgs &, cudaStream_t);
void launch_x_864_0(const XArgs &, cudaStream_t);
void launch_x_864_1(const XArgs &, cudaStream_t);
void launch_x_882_0(const XArgs &, cudaStream_t);
void launch_x_882_1(const XArgs &, cudaStream_t);
void launch_x_896_0(const XArgs &, cudaStream_t);
void launch_x_896_1(const XArgs &, cudaStream_t);
void launch_x_900_0(const XArgs &, cudaStream_t);
void launch_x_900_1(const XArgs &, cudaStream_t);
void launch_x_945_0(const XArgs &, cudaStream_t);
void launch_x_945_1(const XArgs &, cudaStream_t);
void launch_x_960_0(const XArgs &, cudaStream_t);
void launch_x_960_1(const XArgs &, cudaStream_t);
void launch_x_972_0(const XArgs &, cudaStream_t);
void launch_x_972_1(const XArgs &, cudaStream_t);
void launch_x_980_0(const XArgs &, cudaStream_t);
void launch_x_980_1(const XArgs &, cudaStream_t);
void launch_x_1000_0(const XArgs &, cudaStream_t);
void launch_x_1008_0(const XArgs &, cudaStream_t);
void launch_x_1008_1(const XArgs &, cudaStream_t);
void launch_x_1024_0(const XArgs &, cudaStream_t);
void launch_x_1024_1(const XArgs &, cudaStream_t);
void launch_x_1050_0(const XArgs &, cudaStream_t);
void launch_x_1050_1(const XArgs &, cudaStream_t);
void launch_x_1080_0(const XArgs &, cudaStream_t);
void launch_x_1080_1(const XArgs &, cudaStream_t);
void launch_x_1120_0(const XArgs &, cudaStream_t);
void launch_x_1120_1(const XArgs &, cudaStream_t);
void launch_x_1125_0(const XArgs &, cudaStream_t);
void launch_x_1125_1(const XArgs &, cudaStream_t);
void launch_x_1134_0(const XArgs &, cudaStream_t);
void launch_x_1134_1(const XArgs &, cudaStream_t);
void launch_x_1152_0(const XArgs &, cudaStream_t);
void launch_x_1152_1(const XArgs &, cudaStream_t);
void launch_x_1176_0(const XArgs &, cudaStream_t);
void launch_x_1176_1(const XArgs &, cudaStream_t);
void launch_x_1200_0(const XArgs &, cudaStream_t);
void launch_x_1200_1(const XArgs &, cudaStream_t);
void launch_x_1215_0(const XArgs &, cudaStream_t);
void launch_x_1215_1(const XArgs &, cudaStream_t);
void launch_x_1260_0(const XArgs &, cudaStream_t);
void launch_x_1260_1(const XArgs &, cudaStream_t);
void launch_x_1280_0(const XArgs &, cudaStream_t);
void launch_x_1280_1(const XArgs &, cudaStream_t);
void launch_x_1296_0(const XArgs &, cudaStream_t);
void launch_x_1296_1(const XArgs &, cudaStream_t);
void launch_x_1344_0(const XArgs &, cudaStream_t);
void launch_x_1344_1(const XArgs &, cudaStream_t);
void launch_x_1350_0(const XArgs &, cudaStream_t);
void launch_x_1350_1(const XArgs &, cudaStream_t);
void launch_x_1372_0(const XArgs &, cudaStream_t);
void launch_x_1372_1(const XArgs &, cudaStream_t);
void launch_x_1400_0(const XArgs &, cudaStream_t);
void launch_x_1400_1(const XArgs &, cudaStream_t);
void launch_x_1440_0(const XArgs &, cudaStream_t);
void launch_x_1440_1(const XArgs &, cudaStream_t);
void launch_x_1470_0(const XArgs &, cudaStream_t);
void launch_x_1470_1(const XArgs &, cudaStream_t);
void launch_x_1500_0(const XArgs &, cudaStream_t);
void launch_x_1500_1(const XArgs &, cudaStream_t);
void launch_x_1512_0(const XArgs &, cudaStream_t);
void launch_x_1512_1(const XArgs &, cudaStream_t);
void launch_x_1536_0(const XArgs &, cudaStream_t);
void launch_x_1536_1(const XArgs &, cudaStream_t);
void launch_x_1568_0(const XArgs &, cudaStream_t);
void launch_x_1568_1(const XArgs &, cudaStream_t);
void launch_x_1575_0(const XArgs &, cudaStream_t);
void launch_x_1575_1(const XArgs &, cudaStream_t);
void launch_x_1600_0(const XArgs &, cudaStream_t);
void launch_x_1600_1(const XArgs &, cudaStream_t);
void launch_x_1620_0(const XArgs &, cudaStream_t);
void launch_x_1620_1(const XArgs &, cudaStream_t);
void launch_x_1680_0(const XArgs &, cudaStream_t);
void launch_x_1680_1(const XArgs &, cudaStream_t);
void launch_x_1728_0(const XArgs &, cudaStream_t);
void launch_x_1728_1(const XArgs &, cudaStream_t);
void launch_x_1764_0(const XArgs &, cudaStream_t);
void launch_x_1764_1(const XArgs &, cudaStream_t);
void launch_x_1792_0(const XArgs &, cudaStream_t);
void launch_x_1792_1(const XArgs &, cudaStream_t);
void launch_x_1800_0(const XArgs &, cudaStream_t);
void launch_x_1800_1(const XArgs &, cudaStream_t);
void launch_x_1890_0(const XArgs &, cudaStream_t);
void launch_x_1890_1(const XArgs &, cudaStream_t);
void launch_x_1920_0(const XArgs &, cudaStream_t);
void launch_x_1920_1(const XArgs &, cudaStream_t);
void launch_x_1960_0(const XArgs &, cudaStream_t);
void launch_x_1960_1(const XArgs &, cudaStream_t);
void launch_x_2016_0(const XArgs &, cudaStream_t);
void launch_x_2016_1(const XArgs &, cudaStream_t);
void launch_x_2025_0(const XArgs &, cudaStream_t);
void launch_x_2025_1(const XArgs &, cudaStream_t);
void launch_x_2048_0(const XArgs &, cudaStream_t);
void launch_x_2048_1(const XArgs &, cudaStream_t);
void launch_y_2_0(const YArgs &, cudaStream_t);
void launch_y_3_0(const YArgs &, cudaStream_t);
void launch_y_4_0(const YArgs &, cudaStream_t);
void launch_y_4_1(const YArgs &, cudaStream_t);
void launch_y_5_0(const YArgs &, cudaStream_t);
void launch_y_6_0(const YArgs &, cudaStream_t);
void launch_y_6_1(const YArgs &, cudaStream_t);
void launch_y_6_2(const YArgs &, cudaStream_t);
void launch_y_7_0(const YArgs &, cudaStream_t);
void launch_y_8_0(const YArgs &, cudaStream_t);
void launch_y_8_1(const YArgs &, cudaStream_t);
void launch_y_8_2(const YArgs &, cudaStream_t);
void launch_y_9_0(const YArgs &, cudaStream_t);
void launch_y_9_1(const YArgs &, cudaStream_t);
void launch_y_10_0(const YArgs &, cudaStream_t);
void launch_y_10_1(const YArgs &, cudaStream_t);
void launch_y_10_2(const YArgs &, cudaStream_t);
void launch_y_12_0(const YArgs &, cudaStream_t);
void launch_y_12_1(const YArgs &, cudaStream_t);
void launch_y_12_2(const YArgs &, cudaStream_t);
void launch_y_14_0(const YArgs &, cudaStream_t);
void launch_y_14_1(const YArgs &, cudaStream_t);
void launch_y_14_2(const YArgs &, cudaStream_t);
void launch_y_15_0(const YArgs &, cudaStream_t);
void launch_y_15_1(const YArgs &, cudaStream_t);
void launch_y_15_2(const YArgs &, cudaStream_t);
void launch_y_16_0(const YArgs &, cudaStream_t);
void launch_y_16_1(const YArgs &, cudaStream_t);
void launch_y_16_2(const YArgs &, cudaStream_t);
void launch_y_18_0(const YArgs &, cudaStream_t);
void launch_y_18_1(const YArgs &, cudaStream_t);
void launch_y_18_2(const YArgs &, cudaStream_t);
void launch_y_20_0(const YArgs &, cudaStream_t);
void launch_y_20_1(const YArgs &, cudaStream_t);
void launch_y_20_2(const YArgs &, cudaStream_t);
void launch_y_21_0(const YArgs &, cudaStream_t);
void launch_y_21_1(const YArgs &, cudaStream_t);
void launch_y_24_0(const YArgs &, cudaStream_t);
void launch_y_24_1(const YArgs &, cudaStream_t);
void launch_y_24_2(const YArgs &, cudaStream_t);
void launch_y_25_0(const YArgs &, cudaStream_t);
void launch_y_27_0(const YArgs &, cudaStream_t);
void launch_y_27_1(const YArgs &, cudaStream_t);
void launch_y_28_0(const YArgs &, cudaStream_t);
void launch_y_28_1(const YArgs &, cudaStream_t);
void launch_y_28_2(const YArgs &, cudaStream_t);
void launch_y_30_0(const YArgs &, cudaStream_t);
void launch_y_30_1(const YArgs &, cudaStream_t);
void launch_y_30_2(const YArgs &, cudaStream_t);
void launch_y_32_0(const YArgs &, cudaStream_t);
void launch_y_32_1(const YArgs &, cudaStream_t);
void launch_y_32_2(const YArgs &, cudaStream_t);
void launch_y_35_0(const YArgs &, cudaStream_t);
void launch_y_35_1(const YArgs &, cudaStream_t);
void launch_y_36_0(const YArgs &, cudaStream_t);
void launch_y_36_1(const YArgs &, cudaStream_t);
void launch_y_36_2(const YArgs &, cudaStream_t);
void launch_y_40_0(const YArgs &, cudaStream_t);
void launch_y_40_1(const YArgs &, cudaStream_t);
void launch_y_40_2(const YArgs &, cudaStream_t);
void launch_y_42_0(const YArgs &, cudaStream_t);
void launch_y_42_1(const YArgs &, cudaStream_t);
void launch_y_42_2(const YArgs &, cudaStream_t);
void launch_y_45_0(const YArgs &, cudaStream_t);
void launch_y_45_1(const YArgs &, cudaStream_t);
void launch_y_45_2(const YArgs &, cudaStream_t);
void launch_y_48_0(const YArgs &, cudaStream_t);
void launch_y_48_1(const YArgs &, cudaStream_t);
void launch_y_48_2(const YArgs &, cudaStream_t);
void launch_y_49_0(const YArgs &, cudaStream_t);
void launch_y_50_0(const YArgs &, cudaStream_t);
void launch_y_50_1(const YArgs &, cudaStream_t);
void launch_y_50_2(const YArgs &, cudaStream_t);
void launch_y_54_0(const YArgs &, cudaStream_t);
void launch_y_54_1(const YArgs &, cudaStream_t);
void launch_y_54_2(const YArgs &, cudaStream_t);
void launch_y_56_0(const YArgs &, cudaStream_t);
void launch_y_56_1(const YArgs &, cudaStream_t);
void launch_y_56_2(const YArgs &, cudaStream_t);
void launch_y_60_0(const YArgs &, cudaStream_t);
void launch_y_60_1(const YArgs &, cudaStream_t);
void launch_y_60_2(const YArgs &, cudaStream_t);
void launch_y_63_0(const YArgs &, cudaStream_t);
void launch_y_63_1(const YArgs &, cudaStream_t);
void launch_y_63_2(const YArgs &, cudaStream_t);
void launch_y_64_0(const YArgs &, cudaStream_t);
void launch_y_64_1(const YArgs &, cudaStream_t);
void launch_y_64_2(const YArgs &, cudaStream_t);
void launch_y_70_0(const YArgs &, cudaStream_t);
void launch_y_70_1(const YArgs &, cudaStream_t);
void launch_y_70_2(const YArgs &, cudaStream_t);
void launch_y_72_0(const YArgs &, cudaStream_t);
void launch_y_72_1(const YArgs &, cudaStream_t);
void launch_y_72_2(const YArgs &, cudaStream_t);
void launch_y_75_0(const YArgs &, cudaStream_t);
void launch_y_75_1(const YArgs &, cudaStream_t);
void launch_y_75_2(const YArgs &, cudaStream_t);
void launch_y_80_0(const YArgs &, cudaStream_t);
void launch_y_80_1(const YArgs &, cudaStream_t);
void launch_y_80_2(const YArgs &, cudaStream_t);
void launch_y_81_0(const YArgs &, cudaStream_t);
void launch_y_81_1(const YArgs &, cudaStream_t);
void launch_y_84_0(const YArgs &, cudaStream_t);
void launch_y_84_1(const YArgs &, cudaStream_t);
void launch_y_84_2(const YArgs &, cudaStream_t);
void launch_y_90_0(const YArgs &, cudaStream_t);
void launch_y_90_1(const YArgs &, cudaStream_t);
void launch_y_90_2(const YArgs &, cudaStream_t);
void launch_y_96_0(const YArgs &, cudaStream_t);
void launch_y_96_1(const YArgs &, cudaStream_t);
void launch_y_96_2(const YArgs &, cudaStream_t);
void launch_y_98_0(const YArgs &, cudaStream_t);
void launch_y_98_1(const YArgs &, cudaStream_t);
void launch_y_98_2(const YArgs &, cudaStream_t);
void launch_y_100_0(const YArgs &, cudaStream_t);
void launch_y_100_1(const YArgs &, cudaStream_t);
void launch_y_100_2(const YArgs &, cudaStream_t);
void launch_y_105_0(const YArgs &, cudaStream_t);
void launch_y_105_1(const YArgs &, cudaStream_t);
void launch_y_105_2(const YArgs &, cudaStream_t);
void launch_y_108_0(const YArgs &, cudaStream_t);
void launch_y_108_1(const YArgs &, cudaStream_t);
void launch_y_108_2(const YArgs &, cudaStream_t);
void launch_y_112_0(const YArgs &, cudaStream_t);
void launch_y_112_1(const YArgs &, cudaStream_t);
void launch_y_112_2(const YArgs &, cudaStream_t);
void launch_y_120_0(const YArgs &, cudaStream_t);
void launch_y_120_1(const YArgs &, cudaStream_t);
void launch_y_120_2(const YArgs &, cudaStream_t);
void launch_y_125_0(const YArgs &, cudaStream_t);
void launch_y_126_0(const YArgs &, cudaStream_t);
void launch_y_126_1(const YArgs &, cudaStream_t);
void launch_y_126_2(const YArgs &, cudaStream_t);
void launch_y_128_0(const YArgs &, cudaStream_t);
void launch_y_128_1(const YArgs &, cudaStream_t);
void launch_y_128_2(const YArgs &, cudaStream_t);
void launch_y_135_0(const YArgs &, cudaStream_t);
void launch_y_135_1(const YArgs &, cudaStream_t);
void launch_y_135_2(const YArgs &, cudaStream_t);
void launch_y_140_0(const YArgs &, cudaStream_t);
void launch_y_140_1(const YArgs &, cudaStream_t);
void launch_y_140_2(const YArgs &, cudaStream_t);
void launch_y_144_0(const YArgs &, cudaStream_t);
void launch_y_144_1(const YArgs &, cudaStream_t);
void launch_y_144_2(const YArgs &, cudaStream_t);
void launch_y_147_0(const YArgs &, cudaStream_t);
void launch_y_147_1(const YArgs &, cudaStream_t);
void launch_y_150_0(const YArgs &, cudaStream_t);
void launch_y_150_1(const YArgs &, cudaStream_t);
void launch_y_150_2(const YArgs &, cudaStream_t);
void launch_y_160_0(const YArgs &, cudaStream_t);
void launch_y_160_1(const YArgs &, cudaStream_t);
void launch_y_160_2(const YArgs &, cudaStream_t);
void launch_y_162_0(const YArgs &, cudaStream_t);
void launch_y_162_1(const YArgs &, cudaStream_t);
void launch_y_162_2(const YArgs &, cudaStream_t);
void launch_y_168_0(const YArgs &, cudaStream_t);
void launch_y_168_1(const YArgs &, cudaStream_t);
void launch_y_168_2(const YArgs &, cudaStream_t);
void launch_y_175_0(const YArgs &, cudaStream_t);
void launch_y_175_1(const YArgs &, cudaStream_t);
void launch_y_180_0(const YArgs &, cudaStream_t);
void launch_y_180_1(const YArgs &, cudaStream_t);
void launch_y_180_2(const YArgs &, cudaStream_t);
void launch_y_189_0(const YArgs &, cudaStream_t);
void launch_y_189_1(const YArgs &, cudaStream_t);
void launch_y_189_2(const YArgs &, cudaStream_t);
void launch_y_192_0(const YArgs &, cudaStream_t);
void launch_y_192_1(const YArgs &, cudaStream_t);
void launch_y_192_2(const YArgs &, cudaStream_t);
void launch_y_196_0(const YArgs &, cudaStream_t);
void launch_y_196_1(const YArgs &, cudaStream_t);
void launch_y_196_2(const YArgs &, cudaStream_t);
void launch_y_200_0(const YArgs &, cudaStream_t);
void launch_y_200_1(const YArgs &, cudaStream_t);
void launch_y_200_2(const YArgs &, cudaStream_t);
void launch_y_210_0(const YArgs &, cudaStream_t);
void launch_y_210_1(const YArgs &, cudaStream_t);
void launch_y_210_2(const YArgs &, cudaStream_t);
void launch_y_216_0(const YArgs &, cudaStream_t);
void launch_y_216_1(const YArgs &, cudaStream_t);
void launch_y_216_2(const YArgs &, cudaStream_t);
void launch_y_224_0(const YArgs &, cudaStream_t);
void launch_y_224_1(const YArgs &, cudaStream_t);
void launch_y_224_2(const YArgs &, cudaStream_t);
void launch_y_225_0(const YArgs &, cudaStream_t);
void launch_y_225_1(const YArgs &, cudaStream_t);
void launch_y_225_2(const YArgs &, cudaStream_t);
void launch_y_240_0(const YArgs &, cudaStream_t);
void launch_y_240_1(const YArgs &, cudaStream_t);
void launch_y_240_2(const YArgs &, cudaStream_t);
void launch_y_243_0(const YArgs &, cudaStream_t);
void launch_y_243_1(const YArgs &, cudaStream_t);
void launch_y_245_0(const YArgs &, cudaStream_t);
void launch_y_245_1(const YArgs &, cudaStream_t);
void launch_y_250_0(const YArgs &, cudaStream_t);
void launch_y_250_1(const YArgs &, cudaStream_t);
void launch_y_252_0(const YArgs &, cudaStream_t);
void launch_y_252_1(const YArgs &, cudaStream_t);
void launch_y_252_2(const YArgs &, cudaStream_t);
void launch_y_256_0(const YArgs &, cudaStream_t);
void launch_y_256_1(const YArgs &, cudaStream_t);
void launch_y_256_2(const YArgs &, cudaStream_t);
void launch_y_270_0(const YArgs &, cudaStream_t);
void launch_y_270_1(const YArgs &, cudaStream_t);
void launch_y_270_2(const YArgs &, cudaStream_t);
void launch_y_280_0(const YArgs &, cudaStream_t);
void launch_y_280_1(const YArgs &, cudaStream_t);
void launch_y_280_2(const YArgs &, cudaStream_t);
void launch_y_288_0(const YArgs &, cudaStream_t);
void launch_y_288_1(const YArgs &, cudaStream_t);
void launch_y_288_2(const YArgs &, cudaStream_t);
void launch_y_294_0(const YArgs &, cudaStream_t);
void launch_y_294_1(const YArgs &, cudaStream_t);
void launch_y_294_2(const YArgs &, cudaStream_t);
void launch_y_300_0(const YArgs &, cudaStream_t);
void launch_y_300_1(const YArgs &, cudaStream_t);
void launch_y_300_2(const YArgs &, cudaStream_t);
void launch_y_315_0(const YArgs &, cudaStream_t);
void launch_y_315_1(const YArgs &, cudaStream_t);
void launch_y_315_2(const YArgs &, cudaStream_t);
void launch_y_320_0(const YArgs &, cudaStream_t);
void launch_y_320_1(const YArgs &, cudaStream_t);
void launch_y_320_2(const YArgs &, cudaStream_t);
void launch_y_324_0(const YArgs &, cudaStream_t);
void launch_y_324_1(const YArgs &, cudaStream_t);
void launch_y_324_2(const YArgs &, cudaStream_t);
void launch_y_336_0(const YArgs &, cudaStream_t);
void launch_y_336_1(const YArgs &, cudaStream_t);
void launch_y_336_2(const YArgs &, cudaStream_t);
void launch_y_343_0(const YArgs &, cudaStream_t);
void launch_y_350_0(const YArgs &, cudaStream_t);
void launch_y_350_1(const YArgs &, cudaStream_t);
void launch_y_350_2(const YArgs &, cudaStream_t);
void launch_y_360_0(const YArgs &, cudaStream_t);
void launch_y_360_1(const YArgs &, cudaStream_t);
void launch_y_360_2(const YArgs &, cudaStream_t);
void launch_y_375_0(const YArgs &, cudaStream_t);
void launch_y_375_1(const YArgs &, cudaStream_t);
void launch_y_378_0(const YArgs &, cudaStream_t);
void launch_y_378_1(const YArgs &, cudaStream_t);
void launch_y_378_2(const YArgs &, cudaStream_t);
void launch_y_384_0(const YArgs &, cudaStream_t);
void launch_y_384_1(const YArgs &, cudaStream_t);
void launch_y_384_2(const YArgs &, cudaStream_t);
void launch_y_392_0(const YArgs &, cudaStream_t);
void launch_y_392_1(const YArgs &, cudaStream_t);
void launch_y_392_2(const YArgs &, cudaStream_t);
void launch_y_400_0(const YArgs &, cudaStream_t);
void launch_y_400_1(const YArgs &, cudaStream_t);
void launch_y_400_2(const YArgs &, cudaStream_t);
void launch_y_405_0(const YArgs &, cudaStream_t);
void launch_y_405_1(const YArgs &, cudaStream_t);
void launch_y_405_2(const YArgs &, cudaStream_t);
void launch_y_420_0(const YArgs &, cudaStream_t);
void launch_y_420_1(const YArgs &, cudaStream_t);
void launch_y_420_2(const YArgs &, cudaStream_t);
void launch_y_432_0(const YArgs &, cudaStream_t);
void launch_y_432_1(const YArgs &, cudaStream_t);
void launch_y_432_2(const YArgs &, cudaStream_t);
void launch_y_441_0(const YArgs &, cudaStream_t);
void launch_y_441_1(const YArgs &, cudaStream_t);
void launch_y_448_0(const YArgs &, cudaStream_t);
void launch_y_448_1(const YArgs &, cudaStream_t);
void launch_y_448_2(const YArgs &, cudaStream_t);
void launch_y_450_0(const YArgs &, cudaStream_t);
void launch_y_450_1(const YArgs &, cudaStream_t);
void launch_y_450_2(const YArgs &, cudaStream_t);
void launch_y_480_0(const YArgs &, cudaStream_t);
void launch_y_480_1(const YArgs &, cudaStream_t);
void launch_y_480_2(const YArgs &, cudaStream_t);
void launch_y_486_0(const YArgs &, cudaStream_t);
void launch_y_486_1(const YArgs &, cudaStream_t);
void launch_y_490_0(const YArgs &, cudaStream_t);
void launch_y_490_1(const YArgs &, cudaStream_t);
void launch_y_490_2(const YArgs &, cudaStream_t);
void launch_y_500_0(const YArgs &, cudaStream_t);
void launch_y_500_1(const YArgs &, cudaStream_t);
void launch_y_504_0(const YArgs &, cudaStream_t);
void launch_y_504_1(const YArgs &, cudaStream_t);
void launch_y_504_2(const YArgs &, cudaStream_t);
void launch_y_512_0(const YArgs &, cudaStream_t);
void launch_y_512_1(const YArgs &, cudaStream_t);
void launch_y_512_2(const YArgs &, cudaStream_t);
void launch_y_525_0(const YArgs &, cudaStream_t);
void launch_y_525_1(const YArgs &, cudaStream_t);
void launch_y_525_2(const YArgs &, cudaStream_t);
void launch_y_540_0(const YArgs &, cudaStream_t);
void launch_y_540_1(const YArgs &, cudaStream_t);
void launch_y_540_2(const YArgs &, cudaStream_t);
void launch_y_560_0(const YArgs &, cudaStream_t);
void launch_y_560_1(const YArgs &, cudaStream_t);
void launch_y_560_2(const YArgs &, cudaStream_t);
void launch_y_567_0(const YArgs &, cudaStream_t);
void launch_y_567_1(const YArgs &, cudaStream_t);
void launch_y_576_0(const YArgs &, cudaStream_t);
void launch_y_576_1(const YArgs &, cudaStream_t);
void launch_y_576_2(const YArgs &, cudaStream_t);
void launch_y_588_0(const YArgs &, cudaStream_t);
void launch_y_588_1(const YArgs &, cudaStream_t);
void launch_y_588_2(const YArgs &, cudaStream_t);
void launch_y_600_0(const YArgs &, cudaStream_t);
void launch_y_600_1(const YArgs &, cudaStream_t);
void launch_y_600_2(const YArgs &, cudaStream_t);
void launch_y_630_0(const YArgs &, cudaStream_t);
void launch_y_630_1(const YArgs &, cudaStream_t);
void launch_y_630_2(const YArgs &, cudaStream_t);
void launch_y_640_0(const YArgs &, cudaStream_t);
void launch_y_640_1(const YArgs &, cudaStream_t);
void launch_y_640_2(const YArgs &, cudaStream_t);
void launch_y_648_0(const YArgs &, cudaStream_t);
void launch_y_648_1(const YArgs &, cudaStream_t);
void launch_y_648_2(const YArgs &, cudaStream_t);
void launch_y_672_0(const YArgs &, cudaStream_t);
void launch_y_672_1(const YArgs &, cudaStream_t);
void launch_y_672_2(const YArgs &, cudaStream_t);
void launch_y_675_0(const YArgs &, cudaStream_t);
void launch_y_675_1(const YArgs &, cudaStream_t);
void launch_y_675_2(const YArgs &, cudaStream_t);
void launch_y_686_0(const YArgs &, cudaStream_t);
void launch_y_686_1(const YArgs &, cudaStream_t);
void launch_y_700_0(const YArgs &, cudaStream_t);
void launch_y_700_1(const YArgs &, cudaStream_t);
void launch_y_700_2(const YArgs &, cudaStream_t);
void launch_y_720_0(const YArgs &, cudaStream_t);
void launch_y_720_1(const YArgs &, cudaStream_t);
void launch_y_720_2(const YArgs &, cudaStream_t);
void launch_y_729_0(const YArgs &, cudaStream_t);
void launch_y_735_0(const YArgs &, cudaStream_t);
void launch_y_735_1(const YArgs &, cudaStream_t);
void launch_y_750_0(const YArgs &, cudaStream_t);
void launch_y_750_1(const YArgs &, cudaStream_t);
void launch_y_750_2(const YArgs &, cudaStream_t);
void launch_y_756_0(const YArgs &, cudaStream_t);
void launch_y_756_1(const YArgs &, cudaStream_t);
void launch_y_756_2(const YArgs &, cudaStream_t);
void launch_y_768_0(const YArgs &, cudaStream_t);
void launch_y_768_1(const YArgs &, cudaStream_t);
void launch_y_768_2(const YArgs &, cudaStream_t);
void launch_y_784_0(const YArgs &, cudaStream_t);
void launch_y_784_1(const YArgs &, cudaStream_t);
void launch_y_784_2(const YArgs &, cudaStream_t);
void launch_y_800_0(const YArgs &, cudaStream_t);
void launch_y_800_1(const YArgs &, cudaStream_t);
void launch_y_800_2(const YArgs &, cudaStream_t);
void launch_y_810_0(const YArgs &, cudaStream_t);
void launch_y_810_1(const YArgs &, cudaStream_t);
void launch_y_810_2(const YArgs &, cudaStream_t);
void launch_y_840_0(const YArgs &, cudaStream_t);
void launch_y_840_1(const YArgs &, cudaStream_t);
void launch_y_840_2(const YArgs &, cudaStream_t);
void launch_y_864_0(const YArgs &, cudaStream_t);
void launch_y_864_1(const YArgs &, cudaStream_t);
void launch_y_864_2(const YArgs &, cudaStream_t);
void launch_y_882_0(const YArgs &, cudaStream_t);
void launch_y_882_1(const YArgs &, cudaStream_t);
void launch_y_882_2(const YArgs &, cudaStream_t);
void launch_y_896_0(const YArgs &, cudaStream_t);
void launch_y_896_1(const YArgs &, cudaStream_t);
void launch_y_896_2(const YArgs &, cudaStream_t);
void launch_y_900_0(const YArgs &, cudaStream_t);
void launch_y_900_1(const YArgs &, cudaStream_t);
void launch_y_900_2(const YArgs &, cudaStream_t);
void launch_y_945_0(const YArgs &, cudaStream_t);
void launch_y_945_1(const YArgs &, cudaStream_t);
void launch_y_945_2(const YArgs &, cudaStream_t);
void launch_y_960_0(const YArgs &, cudaStream_t);
void launch_y_960_1(const YArgs &, cudaStream_t);
void launch_y_960_2(const YArgs &, cudaStream_t);
void launch_y_972_0(const YArgs &, cudaStream_t);
void launch_y_972_1(const YArgs &, cudaStream_t);
void launch_y_980_0(const YArgs &, cudaStream_t);
void launch_y_980_1(const YArgs &, cudaStream_t);
void launch_y_980_2(const YArgs &, cudaStream_t);
void launch_y_1000_0(const YArgs &, cudaStream_t);
void launch_y_1008_0(const YArgs &, cudaStream_t);
void launch_y_1008_1(const YArgs &, cudaStream_t);
void launch_y_1008_2(const YArgs &, cudaStream_t);
void launch_y_1024_0(const YArgs &, cudaStream_t);
void launch_y_1024_1(const YArgs &, cudaStream_t);
void launch_y_1024_2(const YArgs &, cudaStream_t);
void launch_y_1050_0(const YArgs &, cudaStream_t);
void launch_y_1050_1(const YArgs &, cudaStream_t);
void launch_y_1050_2(const YArgs &, cudaStream_t);
void launch_y_1080_0(const YArgs &, cudaStream_t);
void launch_y_1080_1(const YArgs &, cudaStream_t);
void launch_y_1080_2(const YArgs &, cudaStream_t);
void launch_y_1120_0(const YArgs &, cudaStream_t);
void launch_y_1120_1(const YArgs &, cudaStream_t);
void launch_y_1120_2(const YArgs &, cudaStream_t);
void launch_y_1125_0(const YArgs &, cudaStream_t);
void launch_y_1125_1(const YArgs &, cudaStream_t);
void launch_y_1134_0(const YArgs &, cudaStream_t);
void launch_y_1134_1(const YArgs &, cudaStream_t);
void launch_y_1152_0(const YArgs &, cudaStream_t);
void launch_y_1152_1(const YArgs &, cudaStream_t);
void launch_y_1152_2(const YArgs &, cudaStream_t);
void launch_y_1176_0(const YArgs &, cudaStream_t);
void launch_y_1176_1(const YArgs &, cudaStream_t);
void launch_y_1176_2(const YArgs &, cudaStream_t);
void launch_y_1200_0(const YArgs &, cudaStream_t);
void launch_y_1200_1(const YArgs &, cudaStream_t);
void launch_y_1200_2(const YArgs &, cudaStream_t);
void launch_y_1215_0(const YArgs &, cudaStream_t);
void launch_y_1215_1(const YArgs &, cudaStream_t);
void launch_y_1260_0(const YArgs &, cudaStream_t);
void launch_y_1260_1(const YArgs &, cudaStream_t);
void launch_y_1260_2(const YArgs &, cudaStream_t);
void launch_y_1280_0(const YArgs &, cudaStream_t);
void launch_y_1280_1(const YArgs &, cudaStream_t);
void launch_y_1280_2(const YArgs &, cudaStream_t);
void launch_y_1296_0(const YArgs &, cudaStream_t);
void launch_y_1296_1(const YArgs &, cudaStream_t);
void launch_y_1296_2(const YArgs &, cudaStream_t);
void launch_y_1344_0(const YArgs &, cudaStream_t);
void launch_y_1344_1(const YArgs &, cudaStream_t);
void launch_y_1344_2(const YArgs &, cudaStream_t);
void launch_y_1350_0(const YArgs &, cudaStream_t);
void launch_y_1350_1(const YArgs &, cudaStream_t);
void launch_y_1350_2(const YArgs &, cudaStream_t);
void launch_y_1372_0(const YArgs &, cudaStream_t);
void launch_y_1372_1(const YArgs &, cudaStream_t);
void launch_y_1400_0(const YArgs &, cudaStream_t);
void launch_y_1400_1(const YArgs &, cudaStream_t);
void launch_y_1440_0(const YArgs &, cudaStream_t);
void launch_y_1440_1(const YArgs &, cudaStream_t);
void launch_y_1440_2(const YArgs &, cudaStream_t);
void launch_y_1470_0(const YArgs &, cudaStream_t);
void launch_y_1470_1(const YArgs &, cudaStream_t);
void launch_y_1470_2(const YArgs &, cudaStream_t);
void launch_y_1500_0(const YArgs &, cudaStream_t);
void launch_y_1500_1(const YArgs &, cudaStream_t);
void launch_y_1512_0(const YArgs &, cudaStream_t);
void launch_y_1512_1(const YArgs &, cudaStream_t);
void launch_y_1512_2(const YArgs &, cudaStream_t);
void launch_y_1536_0(const YArgs &, cudaStream_t);
void launch_y_1536_1(const YArgs &, cudaStream_t);
void launch_y_1536_2(const YArgs &, cudaStream_t);
void launch_y_1568_0(const YArgs &, cudaStream_t);
void launch_y_1568_1(const YArgs &, cudaStream_t);
void launch_y_1568_2(const YArgs &, cudaStream_t);
void launch_y_1575_0(const YArgs &, cudaStream_t);
void launch_y_1575_1(const YArgs &, cudaStream_t);
void launch_y_1600_0(const YArgs &, cudaStream_t);
void launch_y_1600_1(const YArgs &, cudaStream_t);
void launch_y_1620_0(const YArgs &, cudaStream_t);
void launch_y_1620_1(const YArgs &, cudaStream_t);
void launch_y_1620_2(const YArgs &, cudaStream_t);
void launch_y_1680_0(const YArgs &, cudaStream_t);
void launch_y_1680_1(const YArgs &, cudaStream_t);
void launch_y_1680_2(const YArgs &, cudaStream_t);
void launch_y_1728_0(const YArgs &, cudaStream_t);
void launch_y_1728_1(const YArgs &, cudaStream_t);
void launch_y_1728_2(const YArgs &, cudaStream_t);
void launch_y_1764_0(const YArgs &, cudaStream_t);
void launch_y_1764_1(const YArgs &, cudaStream_t);
void launch_y_1792_0(const YArgs &, cudaStream_t);
void launch_y_1792_1(const YArgs &, cudaStream_t);
void launch_y_1792_2(const YArgs &, cudaStream_t);
void launch_y_1800_0(const YArgs &, cudaStream_t);
void launch_y_1800_1(const YArgs &, cudaStream_t);
void launch_y_1800_2(const YArgs &, cudaStream_t);
void launch_y_1890_0(const YArgs &, cudaStream_t);
void launch_y_1890_1(const YArgs &, cudaStream_t);
void launch_y_1890_2(const YArgs &, cudaStream_t);
void launch_y_1920_0(const YArgs &, cudaStream_t);
void launch_y_1920_1(const YArgs &, cudaStream_t);
void launch_y_1920_2(const YArgs &, cudaStream_t);
void launch_y_1960_0(const YArgs &, cudaStream_t);
void launch_y_1960_1(const YArgs &, cudaStream_t);
void launch_y_2016_0(const YArgs &, cudaStream_t);
void launch_y_2016_1(const YArgs &, cudaStream_t);
void launch_y_2016_2(const YArgs &, cudaStream_t);
void launch_y_2025_0(const YArgs &, cudaStream_t);
void launch_y_2025_1(const YArgs &, cudaStream_t);
void launch_y_2048_0(const YArgs &, cudaStream_t);
void launch_y_2048_1(const YArgs &, cudaStream_t);
void launch_y_2100_0(const YArgs &, cudaStream_t);
void launch_y_2100_1(const YArgs &, cudaStream_t);
void launch_y_2100_2(const YArgs &, cudaStream_t);
void launch_y_2160_0(const YArgs &, cudaStream_t);
void launch_y_2160_1(const YArgs &, cudaStream_t);
void launch_y_2160_2(const YArgs &, cudaStream_t);
void launch_y_2240_0(const YArgs &, cudaStream_t);
void launch_y_2240_1(const YArgs &, cudaStream_t);
void launch_y_2240_2(const YArgs &, cudaStream_t);
void launch_y_2250_0(const YArgs &, cudaStream_t);
void launch_y_2250_1(const YArgs &, cudaStream_t);
void launch_y_2304_0(const YArgs &, cudaStream_t);
void launch_y_2304_1(const YArgs &, cudaStream_t);
void launch_y_2304_2(const YArgs &, cudaStream_t);
void launch_y_2352_0(const YArgs &, cudaStream_t);
void launch_y_2352_1(const YArgs &, cudaStream_t);
void launch_y_2400_0(const YArgs &, cudaStream_t);
void launch_y_2400_1(const YArgs &, cudaStream_t);
void launch_y_2400_2(const YArgs &, cudaStream_t);
void launch_y_2520_0(const YArgs &, cudaStream_t);
void launch_y_2520_1(const YArgs &, cudaStream_t);
void launch_y_2520_2(const YArgs &, cudaStream_t);
void launch_y_2560_0(const YArgs &, cudaStream_t);
void launch_y_2560_1(const YArgs &, cudaStream_t);
void launch_y_2688_0(const YArgs &, cudaStream_t);
void launch_y_2688_1(const YArgs &, cudaStream_t);
void launch_y_2688_2(const YArgs &, cudaStream_t);
void launch_y_2700_0(const YArgs &, cudaStream_t);
void launch_y_2700_1(const YArgs &, cudaStream_t);
void launch_y_2744_0(const YArgs &, cudaStream_t);
void launch_y_2880_0(const YArgs &, cudaStream_t);
void launch_y_2880_1(const YArgs &, cudaStream_t);
void launch_y_2880_2(const YArgs &, cudaStream_t);
void launch_y_2940_0(const YArgs &, cudaStream_t);
void launch_y_2940_1(const YArgs &, cudaStream_t);
void launch_y_3072_0(const YArgs &, cudaStream_t);
void launch_y_3072_1(const YArgs &, cudaStream_t);
void launch_y_3136_0(const YArgs &, cudaStream_t);
void launch_y_3136_1(const YArgs &, cudaStream_t);
void launch_y_3150_0(const YArgs &, cudaStream_t);
void launch_y_3150_1(const YArgs &, cudaStream_t);
static const LinesPlan kLinesPlans[] = {
    {1, 0, 1, 1, 1, 16, LinesCfg<Rad<1, 1, 1>, 16>::THREADS, LinesCfg<Rad<1, 1, 1>, 16>::SMEM_BYTES, launch_lines_1_0},
    {2, 0, 2, 1, 1, 16, LinesCfg<Rad<2, 1, 1>, 16>::THREADS, LinesCfg<Rad<2, 1, 1>, 16>::SMEM_BYTES, launch_lines_2_0},
    {2, 1, 2, 1, 1, 8, LinesCfg<Rad<2, 1, 1>, 8>::THREADS, LinesCfg<Rad<2, 1, 1>, 8>::SMEM_BYTES, launch_lines_2_1},
    {3, 0, 3, 1, 1, 16, LinesCfg<Rad<3, 1, 1>, 16>::THREADS, LinesCfg<Rad<3, 1, 1>, 16>::SMEM_BYTES, launch_lines_3_0},
    {3, 1, 3, 1, 1, 8, LinesCfg<Rad<3, 1, 1>, 8>::THREADS, LinesCfg<Rad<3, 1, 1>, 8>::SMEM_BYTES, launch_lines_3_1},
    {4, 0, 2, 2, 1, 16, LinesCfg<Rad<2, 2, 1>, 16>::THREADS, LinesCfg<Rad<2, 2, 1>, 16>::SMEM_BYTES, launch_lines_4_0},
    {4, 1, 4, 1, 1, 16, LinesCfg<Rad<4, 1, 1>, 16>::THREADS, LinesCfg<Rad<4, 1, 1>, 16>::SMEM_BYTES, launch_lines_4_1},
    {4, 2, 2, 2, 1, 8, LinesCfg<Rad<2, 2, 1>, 8>::THREADS, LinesCfg<Rad<2, 2, 1>, 8>::SMEM_BYTES, launch_lines_4_2},
    {5, 0, 5, 1, 1, 16, LinesCfg<Rad<5, 1, 1>, 16>::THREADS, LinesCfg<Rad<5, 1, 1>, 16>::SMEM_BYTES, launch_lines_5_0},
    {5, 1, 5, 1, 1, 8, LinesCfg<Rad<5, 1, 1>, 8>::THREADS, LinesCfg<Rad<5, 1, 1>, 8>::SMEM_BYTES, launch_lines_5_1},
    {6, 0, 3, 2, 1, 16, LinesCfg<Rad<3, 2, 1>, 16>::THREADS, LinesCfg<Rad<3, 2, 1>, 16>::SMEM_BYTES, launch_lines_6_0},
    {6, 1, 2, 3, 1, 16, LinesCfg<Rad<2, 3, 1>, 16>::THREADS, LinesCfg<Rad<2, 3, 1>, 16>::SMEM_BYTES, launch_lines_6_1},
    {6, 2, 3, 2, 1, 8, LinesCfg<Rad<3, 2, 1>, 8>::THREADS, LinesCfg<Rad<3, 2, 1>, 8>::SMEM_BYTES, launch_lines_6_2},
    {7, 0, 7, 1, 1, 16, LinesCfg<Rad<7, 1, 1>, 16>::THREADS, LinesCfg<Rad<7, 1, 1>, 16>::SMEM_BYTES, launch_lines_7_0},
    {7, 1, 7, 1, 1, 8, LinesCfg<Rad<7, 1, 1>, 8>::THREADS, LinesCfg<Rad<7, 1, 1>, 8>::SMEM_BYTES, launch_lines_7_1},
    {8, 0, 4, 2, 1, 16, LinesCfg<Rad<4, 2, 1>, 16>::THREADS, LinesCfg<Rad<4, 2, 1>, 16>::SMEM_BYTES, launch_lines_8_0},
    {8, 1, 2, 4, 1, 16, LinesCfg<Rad<2, 4, 1>, 16>::THREADS, LinesCfg<Rad<2, 4, 1>, 16>::SMEM_BYTES, launch_lines_8_1},
    {8, 2, 4, 2, 1, 8, LinesCfg<Rad<4, 2, 1>, 8>::THREADS, LinesCfg<Rad<4, 2, 1>, 8>::SMEM_BYTES, launch_lines_8_2},
    {9, 0, 3, 3, 1, 16, LinesCfg<Rad<3, 3, 1>, 16>::THREADS, LinesCfg<Rad<3, 3, 1>, 16>::SMEM_BYTES, launch_lines_9_0},
    {9, 1, 9, 1, 1, 16, LinesCfg<Rad<9, 1, 1>, 16>::THREADS, LinesCfg<Rad<9, 1, 1>, 16>::SMEM_BYTES, launch_lines_9_1},
    {9, 2, 3, 3, 1, 8, LinesCfg<Rad<3, 3, 1>, 8>::THREADS, LinesCfg<Rad<3, 3, 1>, 8>::SMEM_BYTES, launch_lines_9_2},
    {10, 0, 5, 2, 1, 16, LinesCfg<Rad<5, 2, 1>, 16>::THREADS, LinesCfg<Rad<5, 2, 1>, 16>::SMEM_BYTES, launch_lines_10_0},
    {10, 1, 2, 5, 1, 16, LinesCfg<Rad<2, 5, 1>, 16>::THREADS, LinesCfg<Rad<2, 5, 1>, 16>::SMEM_BYTES, launch_lines_10_1},
    {10, 2, 5, 2, 1, 8, LinesCfg<Rad<5, 2, 1>, 8>::THREADS, LinesCfg<Rad<5, 2, 1>, 8>::SMEM_BYTES, launch_lines_10_2},
    {12, 0, 4, 3, 1, 16, LinesCfg<Rad<4, 3, 1>, 16>::THREADS, LinesCfg<Rad<4, 3, 1>, 16>::SMEM_BYTES, launch_lines_12_0},
    {12, 1, 3, 4, 1, 16, LinesCfg<Rad<3, 4, 1>, 16>::THREADS, LinesCfg<Rad<3, 4, 1>, 16>::SMEM_BYTES, launch_lines_12_1},
    {12, 2, 4, 3, 1, 8, LinesCfg<Rad<4, 3, 1>, 8>::THREADS, LinesCfg<Rad<4, 3, 1>, 8>::SMEM_BYTES, launch_lines_12_2},
    {14, 0, 7, 2, 1, 16, LinesCfg<Rad<7, 2, 1>, 16>::THREADS, LinesCfg<Rad<7, 2, 1>, 16>::SMEM_BYTES, launch_lines_14_0},
    {14, 1, 2, 7, 1, 16, LinesCfg<Rad<2, 7, 1>, 16>::THREADS, LinesCfg<Rad<2, 7, 1>, 16>::SMEM_BYTES, launch_lines_14_1},
    {14, 2, 7, 2, 1, 8, LinesCfg<Rad<7, 2, 1>, 8>::THREADS, LinesCfg<Rad<7, 2, 1>, 8>::SMEM_BYTES, launch_lines_14_2},
    {15, 0, 5, 3, 1, 16, LinesCfg<Rad<5, 3, 1>, 16>::THREADS, LinesCfg<Rad<5, 3, 1>, 16>::SMEM_BYTES, launch_lines_15_0},
    {15, 1, 3, 5, 1, 16, LinesCfg<Rad<3, 5, 1>, 16>::THREADS, LinesCfg<Rad<3, 5, 1>, 16>::SMEM_BYTES, launch_lines_15_1},
    {15, 2, 5, 3, 1, 8, LinesCfg<Rad<5, 3, 1>, 8>::THREADS, LinesCfg<Rad<5, 3, 1>, 8>::SMEM_BYTES, launch_lines_15_2},
    {16, 0, 4, 4, 1, 16, LinesCfg<Rad<4, 4, 1>, 16>::THREADS, LinesCfg<Rad<4, 4, 1>, 16>::SMEM_BYTES, launch_lines_16_0},
    {16, 1, 8, 2, 1, 16, LinesCfg<Rad<8, 2, 1>, 16>::THREADS, LinesCfg<Rad<8, 2, 1>, 16>::SMEM_BYTES, launch_lines_16_1},
    {16, 2, 4, 4, 1, 8, LinesCfg<Rad<4, 4, 1>, 8>::THREADS, LinesCfg<Rad<4, 4, 1>, 8>::SMEM_BYTES, launch_lines_16_2},
    {18, 0, 6, 3, 1, 16, LinesCfg<Rad<6, 3, 1>, 16>::THREADS, LinesCfg<Rad<6, 3, 1>, 16>::SMEM_BYTES, launch_lines_18_0},
    {18, 1, 3, 6, 1, 16, LinesCfg<Rad<3, 6, 1>, 16>::THREADS, LinesCfg<Rad<3, 6, 1>, 16>::SMEM_BYTES, launch_lines_18_1},
    {18, 2, 6, 3, 1, 8, LinesCfg<Rad<6, 3, 1>, 8>::THREADS, LinesCfg<Rad<6, 3, 1>, 8>::SMEM_BYTES, launch_lines_18_2},
    {20, 0, 5, 4, 1, 16, LinesCfg<Rad<5, 4, 1>, 16>::THREADS, LinesCfg<Rad<5, 4, 1>, 16>::SMEM_BYTES, launch_lines_20_0},
    {20, 1, 4, 5, 1, 16, LinesCfg<Rad<4, 5, 1>, 16>::THREADS, LinesCfg<Rad<4, 5, 1>, 16>::SMEM_BYTES, launch_lines_20_1},
    {20, 2, 5, 4, 1, 8, LinesCfg<Rad<5, 4, 1>, 8>::THREADS, LinesCfg<Rad<5, 4, 1>, 8>::SMEM_BYTES, launch_lines_20_2},
    {21, 0, 7, 3, 1, 16, LinesCfg<Rad<7, 3, 1>, 16>::THREADS, LinesCfg<Rad<7, 3, 1>, 16>::SMEM_BYTES, launch_lines_21_0},
    {21, 1, 3, 7, 1, 16, LinesCfg<Rad<3, 7, 1>, 16>::THREADS, LinesCfg<Rad<3, 7, 1>, 16>::SMEM_BYTES, launch_lines_21_1},
    {21, 2, 7, 3, 1, 8, LinesCfg<Rad<7, 3, 1>, 8>::THREADS, LinesCfg<Rad<7, 3, 1>, 8>::SMEM_BYTES, launch_lines_21_2},
    {24, 0, 6, 4, 1, 16, LinesCfg<Rad<6, 4, 1>, 16>::THREADS, LinesCfg<Rad<6, 4, 1>, 16>::SMEM_BYTES, launch_lines_24_0},
    {24, 1, 4, 6, 1, 16, LinesCfg<Rad<4, 6, 1>, 16>::THREADS, LinesCfg<Rad<4, 6, 1>, 16>::SMEM_BYTES, launch_lines_24_1},
    {24, 2, 6, 4, 1, 8, LinesCfg<Rad<6, 4, 1>, 8>::THREADS, LinesCfg<Rad<6, 4, 1>, 8>::SMEM_BYTES, launch_lines_24_2},
    {25, 0, 5, 5, 1, 16, LinesCfg<Rad<5, 5, 1>, 16>::THREADS, LinesCfg<Rad<5, 5, 1>, 16>::SMEM_BYTES, launch_lines_25_0},
    {25, 1, 5, 5, 1, 8, LinesCfg<Rad<5, 5, 1>, 8>::THREADS, LinesCfg<Rad<5, 5, 1>, 8>::SMEM_BYTES, launch_lines_25_1},
    {27, 0, 9, 3, 1, 16, LinesCfg<Rad<9, 3, 1>, 16>::THREADS, LinesCfg<Rad<9, 3, 1>, 16>::SMEM_BYTES, launch_lines_27_0},
    {27, 1, 3, 9, 1, 16, LinesCfg<Rad<3, 9, 1>, 16>::THREADS, LinesCfg<Rad<3, 9, 1>, 16>::SMEM_BYTES, launch_lines_27_1},
    {27, 2, 9, 3, 1, 8, LinesCfg<Rad<9, 3, 1>, 8>::THREADS, LinesCfg<Rad<9, 3, 1>, 8>::SMEM_BYTES, launch_lines_27_2},
    {28, 0, 7, 4, 1, 16, LinesCfg<Rad<7, 4, 1>, 16>::THREADS, LinesCfg<Rad<7, 4, 1>, 16>::SMEM_BYTES, launch_lines_28_0},
    {28, 1, 4, 7, 1, 16, LinesCfg<Rad<4, 7, 1>, 16>::THREADS, LinesCfg<Rad<4, 7, 1>, 16>::SMEM_BYTES, launch_lines_28_1},
    {28, 2, 7, 4, 1, 8, LinesCfg<Rad<7, 4, 1>, 8>::THREADS, LinesCfg<Rad<7, 4, 1>, 8>::SMEM_BYTES, launch_lines_28_2},
    {30, 0, 6, 5, 1, 16, LinesCfg<Rad<6, 5, 1>, 16>::THREADS, LinesCfg<Rad<6, 5, 1>, 16>::SMEM_BYTES, launch_lines_30_0},
    {30, 1, 5, 6, 1, 16, LinesCfg<Rad<5, 6, 1>, 16>::THREADS, LinesCfg<Rad<5, 6, 1>, 16>::SMEM_BYTES, launch_lines_30_1},
    {30, 2, 6, 5, 1, 8, LinesCfg<Rad<6, 5, 1>, 8>::THREADS, LinesCfg<Rad<6, 5, 1>, 8>::SMEM_BYTES, launch_lines_30_2},
    {32, 0, 8, 4, 1, 16, LinesCfg<Rad<8, 4, 1>, 16>::THREADS, LinesCfg<Rad<8, 4, 1>, 16>::SMEM_BYTES, launch_lines_32_0},
    {32, 1, 4, 8, 1, 16, LinesCfg<Rad<4, 8, 1>, 16>::THREADS, LinesCfg<Rad<4, 8, 1>, 16>::SMEM_BYTES, launch_lines_32_1},
    {32, 2, 8, 4, 1, 8, LinesCfg<Rad<8, 4, 1>, 8>::THREADS, LinesCfg<Rad<8, 4, 1>, 8>::SMEM_BYTES, launch_lines_32_2},
    {35, 0, 7, 5, 1, 16, LinesCfg<Rad<7, 5, 1>, 16>::THREADS, LinesCfg<Rad<7, 5, 1>, 16>::SMEM_BYTES, launch_lines_35_0},
    {35, 1, 5, 7, 1, 16, LinesCfg<Rad<5, 7, 1>, 16>::THREADS, LinesCfg<Rad<5, 7, 1>, 16>::SMEM_BYTES, launch_lines_35_1},
    {35, 2, 7, 5, 1, 8, LinesCfg<Rad<7, 5, 1>, 8>::THREADS, LinesCfg<Rad<7, 5, 1>, 8>::SMEM_BYTES, launch_lines_35_2},
    {36, 0, 6, 6, 1, 16, LinesCfg<Rad<6, 6, 1>, 16>::THREADS, LinesCfg<Rad<6, 6, 1>, 16>::SMEM_BYTES, launch_lines_36_0},
    {36, 1, 9, 4, 1, 16, LinesCfg<Rad<9, 4, 1>, 16>::THREADS, LinesCfg<Rad<9, 4, 1>, 16>::SMEM_BYTES, launch_lines_36_1},
    {36, 2, 6, 6, 1, 8, LinesCfg<Rad<6, 6, 1>, 8>::THREADS, LinesCfg<Rad<6, 6, 1>, 8>::SMEM_BYTES, launch_lines_36_2},
    {40, 0, 8, 5, 1, 16, LinesCfg<Rad<8, 5, 1>, 16>::THREADS, LinesCfg<Rad<8, 5, 1>, 16>::SMEM_BYTES, launch_lines_40_0},
    {40, 1, 5, 8, 1, 16, LinesCfg<Rad<5, 8, 1>, 16>::THREADS, LinesCfg<Rad<5, 8, 1>, 16>::SMEM_BYTES, launch_lines_40_1},
    {40, 2, 8, 5, 1, 8, LinesCfg<Rad<8, 5, 1>, 8>::THREADS, LinesCfg<Rad<8, 5, 1>, 8>::SMEM_BYTES, launch_lines_40_2},
    {42, 0, 7, 6, 1, 16, LinesCfg<Rad<7, 6, 1>, 16>::THREADS, LinesCfg<Rad<7, 6, 1>, 16>::SMEM_BYTES, launch_lines_42_0},
    {42, 1, 6, 7, 1, 16, LinesCfg<Rad<6, 7, 1>, 16>::THREADS, LinesCfg<Rad<6, 7, 1>, 16>::SMEM_BYTES, launch_lines_42_1},
    {42, 2, 7, 6, 1, 8, LinesCfg<Rad<7, 6, 1>, 8>::THREADS, LinesCfg<Rad<7, 6, 1>, 8>::SMEM_BYTES, launch_lines_42_2},
    {45, 0, 9, 5, 1, 16, LinesCfg<Rad<9, 5, 1>, 16>::THREADS, LinesCfg<Rad<9, 5, 1>, 16>::SMEM_BYTES, launch_lines_45_0},
    {45, 1, 5, 9, 1, 16, LinesCfg<Rad<5, 9, 1>, 16>::THREADS, LinesCfg<Rad<5, 9, 1>, 16>::SMEM_BYTES, launch_lines_45_1},
    {45, 2, 9, 5, 1, 8, LinesCfg<Rad<9, 5, 1>, 8>::THREADS, LinesCfg<Rad<9, 5, 1>, 8>::SMEM_BYTES, launch_lines_45_2},
    {48, 0, 8, 6, 1, 16, LinesCfg<Rad<8, 6, 1>, 16>::THREADS, LinesCfg<Rad<8, 6, 1>, 16>::SMEM_BYTES, launch_lines_48_0},
    {48, 1, 6, 8, 1, 16, LinesCfg<Rad<6, 8, 1>, 16>::THREADS, LinesCfg<Rad<6, 8, 1>, 16>::SMEM_BYTES, launch_lines_48_1},
    {48, 2, 8, 6, 1, 8, LinesCfg<Rad<8, 6, 1>, 8>::THREADS, LinesCfg<Rad<8, 6, 1>, 8>::SMEM_BYTES, launch_lines_48_2},
    {49, 0, 7, 7, 1, 16, LinesCfg<Rad<7, 7, 1>, 16>::THREADS, LinesCfg<Rad<7, 7, 1>, 16>::SMEM_BYTES, launch_lines_49_0},
    {49, 1, 7, 7, 1, 8, LinesCfg<Rad<7, 7, 1>, 8>::THREADS, LinesCfg<Rad<7, 7, 1>, 8>::SMEM_BYTES, launch_lines_49_1},
    {50, 0, 10, 5, 1, 16, LinesCfg<Rad<10, 5, 1>, 16>::THREADS, LinesCfg<Rad<10, 5, 1>, 16>::SMEM_BYTES, launch_lines_50_0},
    {50, 1, 5, 10, 1, 16, LinesCfg<Rad<5, 10, 1>, 16>::THREADS, LinesCfg<Rad<5, 10, 1>, 16>::SMEM_BYTES, launch_lines_50_1},
    {50, 2, 10, 5, 1, 8, LinesCfg<Rad<10, 5, 1>, 8>::THREADS, LinesCfg<Rad<10, 5, 1>, 8>::SMEM_BYTES, launch_lines_50_2},
    {54, 0, 9, 6, 1, 16, LinesCfg<Rad<9, 6, 1>, 16>::THREADS, LinesCfg<Rad<9, 6, 1>, 16>::SMEM_BYTES, launch_lines_54_0},
    {54, 1, 6, 9, 1, 16, LinesCfg<Rad<6, 9, 1>, 16>::THREADS, LinesCfg<Rad<6, 9, 1>, 16>::SMEM_BYTES, launch_lines_54_1},
    {54, 2, 9, 6, 1, 8, LinesCfg<Rad<9, 6, 1>, 8>::THREADS, LinesCfg<Rad<9, 6, 1>, 8>::SMEM_BYTES, launch_lines_54_2},
    {56, 0, 8, 7, 1, 16, LinesCfg<Rad<8, 7, 1>, 16>::THREADS, LinesCfg<Rad<8, 7, 1>, 16>::SMEM_BYTES, launch_lines_56_0},
    {56, 1, 7, 8, 1, 16, LinesCfg<Rad<7, 8, 1>, 16>::THREADS, LinesCfg<Rad<7, 8, 1>, 16>::SMEM_BYTES, launch_lines_56_1},
    {56, 2, 8, 7, 1, 8, LinesCfg<Rad<8, 7, 1>, 8>::THREADS, LinesCfg<Rad<8, 7, 1>, 8>::SMEM_BYTES, launch_lines_56_2},
    {60, 0, 10, 6, 1, 16, LinesCfg<Rad<10, 6, 1>, 16>::THREADS, LinesCfg<Rad<10, 6, 1>, 16>::SMEM_BYTES, launch_lines_60_0},
    {60, 1, 6, 10, 1, 16, LinesCfg<Rad<6, 10, 1>, 16>::THREADS, LinesCfg<Rad<6, 10, 1>, 16>::SMEM_BYTES, launch_lines_60_1},
    {60, 2, 10, 6, 1, 8, LinesCfg<Rad<10, 6, 1>, 8>::THREADS, LinesCfg<Rad<10, 6, 1>, 8>::SMEM_BYTES, launch_lines_60_2},
    {63, 0, 9, 7, 1, 16, LinesCfg<Rad<9, 7, 1>, 16>::THREADS, LinesCfg<Rad<9, 7, 1>, 16>::SMEM_BYTES, launch_lines_63_0},
    {63, 1, 7, 9, 1, 16, LinesCfg<Rad<7, 9, 1>, 16>::THREADS, LinesCfg<Rad<7, 9, 1>, 16>::SMEM_BYTES, launch_lines_63_1},
    {63, 2, 9, 7, 1, 8, LinesCfg<Rad<9, 7, 1>, 8>::THREADS, LinesCfg<Rad<9, 7, 1>, 8>::SMEM_BYTES, launch_lines_63_2},
    {64, 0, 8, 8, 1, 16, LinesCfg<Rad<8, 8, 1>, 16>::THREADS, LinesCfg<Rad<8, 8, 1>, 16>::SMEM_BYTES, launch_lines_64_0},
    {64, 1, 16, 4, 1, 16, LinesCfg<Rad<16, 4, 1>, 16>::THREADS, LinesCfg<Rad<16, 4, 1>, 16>::SMEM_BYTES, launch_lines_64_1},
    {64, 2, 8, 8, 1, 8, LinesCfg<Rad<8, 8, 1>, 8>::THREADS, LinesCfg<Rad<8, 8, 1>, 8>::SMEM_BYTES, launch_lines_64_2},
    {70, 0, 10, 7, 1, 16, LinesCfg<Rad<10, 7, 1>, 16>::THREADS, LinesCfg<Rad<10, 7, 1>, 16>::SMEM_BYTES, launch_lines_70_0},
    {70, 1, 7, 10, 1, 16, LinesCfg<Rad<7, 10, 1>, 16>::THREADS, LinesCfg<Rad<7, 10, 1>, 16>::SMEM_BYTES, launch_lines_70_1},
    {70, 2, 10, 7, 1, 8, LinesCfg<Rad<10, 7, 1>, 8>::THREADS, LinesCfg<Rad<10, 7, 1>, 8>::SMEM_BYTES, launch_lines_70_2},
    {72, 0, 9, 8, 1, 16, LinesCfg<Rad<9, 8, 1>, 16>::THREADS, LinesCfg<Rad<9, 8, 1>, 16>::SMEM_BYTES, launch_lines_72_0},
    {72, 1, 8, 9, 1, 16, LinesCfg<Rad<8, 9, 1>, 16>::THREADS, LinesCfg<Rad<8, 9, 1>, 16>::SMEM_BYTES, launch_lines_72_1},
    {72, 2, 9, 8, 1, 8, LinesCfg<Rad<9, 8, 1>, 8>::THREADS, LinesCfg<Rad<9, 8, 1>, 8>::SMEM_BYTES, launch_lines_72_2},
    {75, 0, 15, 5, 1, 16, LinesCfg<Rad<15, 5, 1>, 16>::THREADS, LinesCfg<Rad<15, 5, 1>, 16>::SMEM_BYTES, launch_lines_75_0},
    {75, 1, 5, 15, 1, 16, LinesCfg<Rad<5, 15, 1>, 16>::THREADS, LinesCfg<Rad<5, 15, 1>, 16>::SMEM_BYTES, launch_lines_75_1},
    {75, 2, 15, 5, 1, 8, LinesCfg<Rad<15, 5, 1>, 8>::THREADS, LinesCfg<Rad<15, 5, 1>, 8>::SMEM_BYTES, launch_lines_75_2},
    {80, 0, 10, 8, 1, 16, LinesCfg<Rad<10, 8, 1>, 16>::THREADS, LinesCfg<Rad<10, 8, 1>, 16>::SMEM_BYTES, launch_lines_80_0},
    {80, 1, 8, 10, 1, 16, LinesCfg<Rad<8, 10, 1>, 16>::THREADS, LinesCfg<Rad<8, 10, 1>, 16>::SMEM_BYTES, launch_lines_80_1},
    {80, 2, 10, 8, 1, 8, LinesCfg<Rad<10, 8, 1>, 8>::THREADS, LinesCfg<Rad<10, 8, 1>, 8>::SMEM_BYTES, launch_lines_80_2},
    {81, 0, 9, 9, 1, 16, LinesCfg<Rad<9, 9, 1>, 16>::THREADS, LinesCfg<Rad<9, 9, 1>, 16>::SMEM_BYTES, launch_lines_81_0},
    {81, 1, 3, 3, 9, 16, LinesCfg<Rad<3, 3, 9>, 16>::THREADS, LinesCfg<Rad<3, 3, 9>, 16>::SMEM_BYTES, launch_lines_81_1},
    {81, 2, 9, 9, 1, 8, LinesCfg<Rad<9, 9, 1>, 8>::THREADS, LinesCfg<Rad<9, 9, 1>, 8>::SMEM_BYTES, launch_lines_81_2},
    {84, 0, 12, 7, 1, 16, LinesCfg<Rad<12, 7, 1>, 16>::THREADS, LinesCfg<Rad<12, 7, 1>, 16>::SMEM_BYTES, launch_lines_84_0},
    {84, 1, 7, 12, 1, 16, LinesCfg<Rad<7, 12, 1>, 16>::THREADS, LinesCfg<Rad<7, 12, 1>, 16>::SMEM_BYTES, launch_lines_84_1},
    {84, 2, 12, 7, 1, 8, LinesCfg<Rad<12, 7, 1>, 8>::THREADS, LinesCfg<Rad<12, 7, 1>, 8>::SMEM_BYTES, launch_lines_84_2},
    {90, 0, 10, 9, 1, 16, LinesCfg<Rad<10, 9, 1>, 16>::THREADS, LinesCfg<Rad<10, 9, 1>, 16>::SMEM_BYTES, launch_lines_90_0},
    {90, 1, 9, 10, 1, 16, LinesCfg<Rad<9, 10, 1>, 16>::THREADS, LinesCfg<Rad<9, 10, 1>, 16>::SMEM_BYTES, launch_lines_90_1},
    {90, 2, 10, 9, 1, 8, LinesCfg<Rad<10, 9, 1>, 8>::THREADS, LinesCfg<Rad<10, 9, 1>, 8>::SMEM_BYTES, launch_lines_90_2},
    {96, 0, 12, 8, 1, 16, LinesCfg<Rad<12, 8, 1>, 16>::THREADS, LinesCfg<Rad<12, 8, 1>, 16>::SMEM_BYTES, launch_lines_96_0},
    {96, 1, 8, 12, 1, 16, LinesCfg<Rad<8, 12, 1>, 16>::THREADS, LinesCfg<Rad<8, 12, 1>, 16>::SMEM_BYTES, launch_lines_96_1},
    {96, 2, 12, 8, 1, 8, LinesCfg<Rad<12, 8, 1>, 8>::THREADS, LinesCfg<Rad<12, 8, 1>, 8>::SMEM_BYTES, launch_lines_96_2},
    {98, 0, 14, 7, 1, 16, LinesCfg<Rad<14, 7, 1>, 16>::THREADS, LinesCfg<Rad<14, 7, 1>, 16>::SMEM_BYTES, launch_lines_98_0},
    {98, 1, 7, 14, 1, 16, LinesCfg<Rad<7, 14, 1>, 16>::THREADS, LinesCfg<Rad<7, 14, 1>, 16>::SMEM_BYTES, launch_lines_98_1},
    {98, 2, 14, 7, 1, 8, LinesCfg<Rad<14, 7, 1>, 8>::THREADS, LinesCfg<Rad<14, 7, 1>, 8>::SMEM_BYTES, launch_lines_98_2},
    {100, 0, 10, 10, 1, 16, LinesCfg<Rad<10, 10, 1>, 16>::THREADS, LinesCfg<Rad<10, 10, 1>, 16>::SMEM_BYTES, launch_lines_100_0},
    {100, 1, 5, 4, 5, 16, LinesCfg<Rad<5, 4, 5>, 16>::THREADS, LinesCfg<Rad<5, 4, 5>, 16>::SMEM_BYTES, launch_lines_100_1},
    {100, 2, 10, 10, 1, 8, LinesCfg<Rad<10, 10, 1>, 8>::THREADS, LinesCfg<Rad<10, 10, 1>, 8>::SMEM_BYTES, launch_lines_100_2},
    {105, 0, 15, 7, 1, 16, LinesCfg<Rad<15, 7, 1>, 16>::THREADS, LinesCfg<Rad<15, 7, 1>, 16>::SMEM_BYTES, launch_lines_105_0},
    {105, 1, 7, 15, 1, 16, LinesCfg<Rad<7, 15, 1>, 16>::THREADS, LinesCfg<Rad<7, 15, 1>, 16>::SMEM_BYTES, launch_lines_105_1},
    {105, 2, 15, 7, 1, 8, LinesCfg<Rad<15, 7, 1>, 8>::THREADS, LinesCfg<Rad<15, 7, 1>, 8>::SMEM_BYTES, launch_lines_105_2},
    {108, 0, 12, 9, 1, 16, LinesCfg<Rad<12, 9, 1>, 16>::THREADS, LinesCfg<Rad<12, 9, 1>, 16>::SMEM_BYTES, launch_lines_108_0},
    {108, 1, 9, 12, 1, 16, LinesCfg<Rad<9, 12, 1>, 16>::THREADS, LinesCfg<Rad<9, 12, 1>, 16>::SMEM_BYTES, launch_lines_108_1},
    {108, 2, 12, 9, 1, 8, LinesCfg<Rad<12, 9, 1>, 8>::THREADS, LinesCfg<Rad<12, 9, 1>, 8>::SMEM_BYTES, launch_lines_108_2},
    {112, 0, 14, 8, 1, 16, LinesCfg<Rad<14, 8, 1>, 16>::THREADS, LinesCfg<Rad<14, 8, 1>, 16>::SMEM_BYTES, launch_lines_112_0},
    {112, 1, 8, 14, 1, 16, LinesCfg<Rad<8, 14, 1>, 16>::THREADS, LinesCfg<Rad<8, 14, 1>, 16>::SMEM_BYTES, launch_lines_112_1},
    {112, 2, 14, 8, 1, 8, LinesCfg<Rad<14, 8, 1>, 8>::THREADS, LinesCfg<Rad<14, 8, 1>, 8>::SMEM_BYTES, launch_lines_112_2},
    {120, 0, 12, 10, 1, 16, LinesCfg<Rad<12, 10, 1>, 16>::THREADS, LinesCfg<Rad<12, 10, 1>, 16>::SMEM_BYTES, launch_lines_120_0},
    {120, 1, 10, 12, 1, 16, LinesCfg<Rad<10, 12, 1>, 16>::THREADS, LinesCfg<Rad<10, 12, 1>, 16>::SMEM_BYTES, launch_lines_120_1},
    {120, 2, 12, 10, 1, 8, LinesCfg<Rad<12, 10, 1>, 8>::THREADS, LinesCfg<Rad<12, 10, 1>, 8>::SMEM_BYTES, launch_lines_120_2},
    {125, 0, 5, 5, 5, 16, LinesCfg<Rad<5, 5, 5>, 16>::THREADS, LinesCfg<Rad<5, 5, 5>, 16>::SMEM_BYTES, launch_lines_125_0},
    {125, 1, 5, 5, 5, 8, LinesCfg<Rad<5, 5, 5>, 8>::THREADS, LinesCfg<Rad<5, 5, 5>, 8>::SMEM_BYTES, launch_lines_125_1},
    {126, 0, 14, 9, 1, 16, LinesCfg<Rad<14, 9, 1>, 16>::THREADS, LinesCfg<Rad<14, 9, 1>, 16>::SMEM_BYTES, launch_lines_126_0},
    {126, 1, 9, 14, 1, 16, LinesCfg<Rad<9, 14, 1>, 16>::THREADS, LinesCfg<Rad<9, 14, 1>, 16>::SMEM_BYTES, launch_lines_126_1},
    {126, 2, 14, 9, 1, 8, LinesCfg<Rad<14, 9, 1>, 8>::THREADS, LinesCfg<Rad<14, 9, 1>, 8>::SMEM_BYTES, launch_lines_126_2},
    {128, 0, 16, 8, 1, 16, LinesCfg<Rad<16, 8, 1>, 16>::THREADS, LinesCfg<Rad<16, 8, 1>, 16>::SMEM_BYTES, launch_lines_128_0},
    {128, 1, 8, 16, 1, 16, LinesCfg<Rad<8, 16, 1>, 16>::THREADS, LinesCfg<Rad<8, 16, 1>, 16>::SMEM_BYTES, launch_lines_128_1},
    {128, 2, 16, 8, 1, 8, LinesCfg<Rad<16, 8, 1>, 8>::THREADS, LinesCfg<Rad<16, 8, 1>, 8>::SMEM_BYTES, launch_lines_128_2},
    {135, 0, 15, 9, 1, 16, LinesCfg<Rad<15, 9, 1>, 16>::THREADS, LinesCfg<Rad<15, 9, 1>, 16>::SMEM_BYTES, launch_lines_135_0},
    {135, 1, 9, 15, 1, 16, LinesCfg<Rad<9, 15, 1>, 16>::THREADS, LinesCfg<Rad<9, 15, 1>, 16>::SMEM_BYTES, launch_lines_135_1},
    {135, 2, 15, 9, 1, 8, LinesCfg<Rad<15, 9, 1>, 8>::THREADS, LinesCfg<Rad<15, 9, 1>, 8>::SMEM_BYTES, launch_lines_135_2},
    {140, 0, 14, 10, 1, 16, LinesCfg<Rad<14, 10, 1>, 16>::THREADS, LinesCfg<Rad<14, 10, 1>, 16>::SMEM_BYTES, launch_lines_140_0},
    {140, 1, 10, 14, 1, 16, LinesCfg<Rad<10, 14, 1>, 16>::THREADS, LinesCfg<Rad<10, 14, 1>, 16>::SMEM_BYTES, launch_lines_140_1},
    {140, 2, 14, 10, 1, 8, LinesCfg<Rad<14, 10, 1>, 8>::THREADS, LinesCfg<Rad<14, 10, 1>, 8>::SMEM_BYTES, launch_lines_140_2},
    {144, 0, 12, 12, 1, 16, LinesCfg<Rad<12, 12, 1>, 16>::THREADS, LinesCfg<Rad<12, 12, 1>, 16>::SMEM_BYTES, launch_lines_144_0},
    {144, 1, 16, 9, 1, 16, LinesCfg<Rad<16, 9, 1>, 16>::THREADS, LinesCfg<Rad<16, 9, 1>, 16>::SMEM_BYTES, launch_lines_144_1},
    {144, 2, 12, 12, 1, 8, LinesCfg<Rad<12, 12, 1>, 8>::THREADS, LinesCfg<Rad<12, 12, 1>, 8>::SMEM_BYTES, launch_lines_144_2},
    {147, 0, 7, 3, 7, 16, LinesCfg<Rad<7, 3, 7>, 16>::THREADS, LinesCfg<Rad<7, 3, 7>, 16>::SMEM_BYTES, launch_lines_147_0},
    {147, 1, 3, 7, 7, 16, LinesCfg<Rad<3, 7, 7>, 16>::THREADS, LinesCfg<Rad<3, 7, 7>, 16>::SMEM_BYTES, launch_lines_147_1},
    {147, 2, 7, 3, 7, 8, LinesCfg<Rad<7, 3, 7>, 8>::THREADS, LinesCfg<Rad<7, 3, 7>, 8>::SMEM_BYTES, launch_lines_147_2},
    {150, 0, 15, 10, 1, 16, LinesCfg<Rad<15, 10, 1>, 16>::THREADS, LinesCfg<Rad<15, 10, 1>, 16>::SMEM_BYTES, launch_lines_150_0},
    {150, 1, 10, 15, 1, 16, LinesCfg<Rad<10, 15, 1>, 16>::THREADS, LinesCfg<Rad<10, 15, 1>, 16>::SMEM_BYTES, launch_lines_150_1},
    {150, 2, 15, 10, 1, 8, LinesCfg<Rad<15, 10, 1>, 8>::THREADS, LinesCfg<Rad<15, 10, 1>, 8>::SMEM_BYTES, launch_lines_150_2},
    {160, 0, 16, 10, 1, 16, LinesCfg<Rad<16, 10, 1>, 16>::THREADS, LinesCfg<Rad<16, 10, 1>, 16>::SMEM_BYTES, launch_lines_160_0},
    {160, 1, 10, 16, 1, 16, LinesCfg<Rad<10, 16, 1>, 16>::THREADS, LinesCfg<Rad<10, 16, 1>, 16>::SMEM_BYTES, launch_lines_160_1},
    {160, 2, 16, 10, 1, 8, LinesCfg<Rad<16, 10, 1>, 8>::THREADS, LinesCfg<Rad<16, 10, 1>, 8>::SMEM_BYTES, launch_lines_160_2},
    {162, 0, 9, 3, 6, 16, LinesCfg<Rad<9, 3, 6>, 16>::THREADS, LinesCfg<Rad<9, 3, 6>, 16>::SMEM_BYTES, launch_lines_162_0},
    {162, 1, 6, 3, 9, 16, LinesCfg<Rad<6, 3, 9>, 16>::THREADS, LinesCfg<Rad<6, 3, 9>, 16>::SMEM_BYTES, launch_lines_162_1},
    {162, 2, 9, 3, 6, 8, LinesCfg<Rad<9, 3, 6>, 8>::THREADS, LinesCfg<Rad<9, 3, 6>, 8>::SMEM_BYTES, launch_lines_162_2},
    {168, 0, 14, 12, 1, 16, LinesCfg<Rad<14, 12, 1>, 16>::THREADS, LinesCfg<Rad<14, 12, 1>, 16>::SMEM_BYTES, launch_lines_168_0},
    {168, 1, 12, 14, 1, 16, LinesCfg<Rad<12, 14, 1>, 16>::THREADS, LinesCfg<Rad<12, 14, 1>, 16>::SMEM_BYTES, launch_lines_168_1},
    {168, 2, 14, 12, 1, 8, LinesCfg<Rad<14, 12, 1>, 8>::THREADS, LinesCfg<Rad<14, 12, 1>, 8>::SMEM_BYTES, launch_lines_168_2},
    {175, 0, 7, 5, 5, 16, LinesCfg<Rad<7, 5, 5>, 16>::THREADS, LinesCfg<Rad<7, 5, 5>, 16>::SMEM_BYTES, launch_lines_175_0},
    {175, 1, 5, 5, 7, 16, LinesCfg<Rad<5, 5, 7>, 16>::THREADS, LinesCfg<Rad<5, 5, 7>, 16>::SMEM_BYTES, launch_lines_175_1},
    {175, 2, 7, 5, 5, 8, LinesCfg<Rad<7, 5, 5>, 8>::THREADS, LinesCfg<Rad<7, 5, 5>, 8>::SMEM_BYTES, launch_lines_175_2},
    {180, 0, 15, 12, 1, 16, LinesCfg<Rad<15, 12, 1>, 16>::THREADS, LinesCfg<Rad<15, 12, 1>, 16>::SMEM_BYTES, launch_lines_180_0},
    {180, 1, 12, 15, 1, 16, LinesCfg<Rad<12, 15, 1>, 16>::THREADS, LinesCfg<Rad<12, 15, 1>, 16>::SMEM_BYTES, launch_lines_180_1},
    {180, 2, 15, 12, 1, 8, LinesCfg<Rad<15, 12, 1>, 8>::THREADS, LinesCfg<Rad<15, 12, 1>, 8>::SMEM_BYTES, launch_lines_180_2},
    {189, 0, 9, 3, 7, 16, LinesCfg<Rad<9, 3, 7>, 16>::THREADS, LinesCfg<Rad<9, 3, 7>, 16>::SMEM_BYTES, launch_lines_189_0},
    {189, 1, 7, 3, 9, 16, LinesCfg<Rad<7, 3, 9>, 16>::THREADS, LinesCfg<Rad<7, 3, 9>, 16>::SMEM_BYTES, launch_lines_189_1},
    {189, 2, 9, 3, 7, 8, LinesCfg<Rad<9, 3, 7>, 8>::THREADS, LinesCfg<Rad<9, 3, 7>, 8>::SMEM_BYTES, launch_lines_189_2},
    {192, 0, 16, 12, 1, 16, LinesCfg<Rad<16, 12, 1>, 16>::THREADS, LinesCfg<Rad<16, 12, 1>, 16>::SMEM_BYTES, launch_lines_192_0},
    {192, 1, 12, 16, 1, 16, LinesCfg<Rad<12, 16, 1>, 16>::THREADS, LinesCfg<Rad<12, 16, 1>, 16>::SMEM_BYTES, launch_lines_192_1},
    {192, 2, 16, 12, 1, 8, LinesCfg<Rad<16, 12, 1>, 8>::THREADS, LinesCfg<Rad<16, 12, 1>, 8>::SMEM_BYTES, launch_lines_192_2},
    {196, 0, 14, 14, 1, 16, LinesCfg<Rad<14, 14, 1>, 16>::THREADS, LinesCfg<Rad<14, 14, 1>, 16>::SMEM_BYTES, launch_lines_196_0},
    {196, 1, 7, 4, 7, 16, LinesCfg<Rad<7, 4, 7>, 16>::THREADS, LinesCfg<Rad<7, 4, 7>, 16>::SMEM_BYTES, launch_lines_196_1},
    {196, 2, 14, 14, 1, 8, LinesCfg<Rad<14, 14, 1>, 8>::THREADS, LinesCfg<Rad<14, 14, 1>, 8>::SMEM_BYTES, launch_lines_196_2},
    {200, 0, 8, 5, 5, 16, LinesCfg<Rad<8, 5, 5>, 16>::THREADS, LinesCfg<Rad<8, 5, 5>, 16>::SMEM_BYTES, launch_lines_200_0},
    {200, 1, 5, 5, 8, 16, LinesCfg<Rad<5, 5, 8>, 16>::THREADS, LinesCfg<Rad<5, 5, 8>, 16>::SMEM_BYTES, launch_lines_200_1},
    {200, 2, 8, 5, 5, 8, LinesCfg<Rad<8, 5, 5>, 8>::THREADS, LinesCfg<Rad<8, 5, 5>, 8>::SMEM_BYTES, launch_lines_200_2},
    {210, 0, 15, 14, 1, 16, LinesCfg<Rad<15, 14, 1>, 16>::THREADS, LinesCfg<Rad<15, 14, 1>, 16>::SMEM_BYTES, launch_lines_210_0},
    {210, 1, 14, 15, 1, 16, LinesCfg<Rad<14, 15, 1>, 16>::THREADS, LinesCfg<Rad<14, 15, 1>, 16>::SMEM_BYTES, launch_lines_210_1},
    {210, 2, 15, 14, 1, 8, LinesCfg<Rad<15, 14, 1>, 8>::THREADS, LinesCfg<Rad<15, 14, 1>, 8>::SMEM_BYTES, launch_lines_210_2},
    {216, 0, 6, 6, 6, 16, LinesCfg<Rad<6, 6, 6>, 16>::THREADS, LinesCfg<Rad<6, 6, 6>, 16>::SMEM_BYTES, launch_lines_216_0},
    {216, 1, 9, 4, 6, 16, LinesCfg<Rad<9, 4, 6>, 16>::THREADS, LinesCfg<Rad<9, 4, 6>, 16>::SMEM_BYTES, launch_lines_216_1},
    {216, 2, 6, 6, 6, 8, LinesCfg<Rad<6, 6, 6>, 8>::THREADS, LinesCfg<Rad<6, 6, 6>, 8>::SMEM_BYTES, launch_lines_216_2},
    {224, 0, 16, 14, 1, 16, LinesCfg<Rad<16, 14, 1>, 16>::THREADS, LinesCfg<Rad<16, 14, 1>, 16>::SMEM_BYTES, launch_lines_224_0},
    {224, 1, 14, 16, 1, 16, LinesCfg<Rad<14, 16, 1>, 16>::THREADS, LinesCfg<Rad<14, 16, 1>, 16>::SMEM_BYTES, launch_lines_224_1},
    {224, 2, 16, 14, 1, 8, LinesCfg<Rad<16, 14, 1>, 8>::THREADS, LinesCfg<Rad<16, 14, 1>, 8>::SMEM_BYTES, launch_lines_224_2},
    {225, 0, 15, 15, 1, 16, LinesCfg<Rad<15, 15, 1>, 16>::THREADS, LinesCfg<Rad<15, 15, 1>, 16>::SMEM_BYTES, launch_lines_225_0},
    {225, 1, 9, 5, 5, 16, LinesCfg<Rad<9, 5, 5>, 16>::THREADS, LinesCfg<Rad<9, 5, 5>, 16>::SMEM_BYTES, launch_lines_225_1},
    {225, 2, 15, 15, 1, 8, LinesCfg<Rad<15, 15, 1>, 8>::THREADS, LinesCfg<Rad<15, 15, 1>, 8>::SMEM_BYTES, launch_lines_225_2},
    {240, 0, 16, 15, 1, 16, LinesCfg<Rad<16, 15, 1>, 16>::THREADS, LinesCfg<Rad<16, 15, 1>, 16>::SMEM_BYTES, launch_lines_240_0},
    {240, 1, 15, 16, 1, 16, LinesCfg<Rad<15, 16, 1>, 16>::THREADS, LinesCfg<Rad<15, 16, 1>, 16>::SMEM_BYTES, launch_lines_240_1},
    {240, 2, 16, 15, 1, 8, LinesCfg<Rad<16, 15, 1>, 8>::THREADS, LinesCfg<Rad<16, 15, 1>, 8>::SMEM_BYTES, launch_lines_240_2},
    {243, 0, 9, 3, 9, 8, LinesCfg<Rad<9, 3, 9>, 8>::THREADS, LinesCfg<Rad<9, 3, 9>, 8>::SMEM_BYTES, launch_lines_243_0},
    {243, 1, 3, 9, 9, 8, LinesCfg<Rad<3, 9, 9>, 8>::THREADS, LinesCfg<Rad<3, 9, 9>, 8>::SMEM_BYTES, launch_lines_243_1},
    {243, 2, 9, 3, 9, 4, LinesCfg<Rad<9, 3, 9>, 4>::THREADS, LinesCfg<Rad<9, 3, 9>, 4>::SMEM_BYTES, launch_lines_243_2},
    {245, 0, 7, 5, 7, 16, LinesCfg<Rad<7, 5, 7>, 16>::THREADS, LinesCfg<Rad<7, 5, 7>, 16>::SMEM_BYTES, launch_lines_245_0},
    {245, 1, 5, 7, 7, 16, LinesCfg<Rad<5, 7, 7>, 16>::THREADS, LinesCfg<Rad<5, 7, 7>, 16>::SMEM_BYTES, launch_lines_245_1},
    {245, 2, 7, 5, 7, 8, LinesCfg<Rad<7, 5, 7>, 8>::THREADS, LinesCfg<Rad<7, 5, 7>, 8>::SMEM_BYTES, launch_lines_245_2},
    {250, 0, 10, 5, 5, 16, LinesCfg<Rad<10, 5, 5>, 16>::THREADS, LinesCfg<Rad<10, 5, 5>, 16>::SMEM_BYTES, launch_lines_250_0},
    {250, 1, 5, 5, 10, 16, LinesCfg<Rad<5, 5, 10>, 16>::THREADS, LinesCfg<Rad<5, 5, 10>, 16>::SMEM_BYTES, launch_lines_250_1},
    {250, 2, 10, 5, 5, 8, LinesCfg<Rad<10, 5, 5>, 8>::THREADS, LinesCfg<Rad<10, 5, 5>, 8>::SMEM_BYTES, launch_lines_250_2},
    {252, 0, 7, 6, 6, 16, LinesCfg<Rad<7, 6, 6>, 16>::THREADS, LinesCfg<Rad<7, 6, 6>, 16>::SMEM_BYTES, launch_lines_252_0},
    {252, 1, 6, 6, 7, 16, LinesCfg<Rad<6, 6, 7>, 16>::THREADS, LinesCfg<Rad<6, 6, 7>, 16>::SMEM_BYTES, launch_lines_252_1},
    {252, 2, 7, 6, 6, 8, LinesCfg<Rad<7, 6, 6>, 8>::THREADS, LinesCfg<Rad<7, 6, 6>, 8>::SMEM_BYTES, launch_lines_252_2},
    {256, 0, 16, 16, 1, 16, LinesCfg<Rad<16, 16, 1>, 16>::THREADS, LinesCfg<Rad<16, 16, 1>, 16>::SMEM_BYTES, launch_lines_256_0},
    {256, 1, 8, 4, 8, 16, LinesCfg<Rad<8, 4, 8>, 16>::THREADS, LinesCfg<Rad<8, 4, 8>, 16>::SMEM_BYTES, launch_lines_256_1},
    {256, 2, 16, 16, 1, 8, LinesCfg<Rad<16, 16, 1>, 8>::THREADS, LinesCfg<Rad<16, 16, 1>, 8>::SMEM_BYTES, launch_lines_256_2},
    {270, 0, 9, 5, 6, 16, LinesCfg<Rad<9, 5, 6>, 16>::THREADS, LinesCfg<Rad<9, 5, 6>, 16>::SMEM_BYTES, launch_lines_270_0},
    {270, 1, 6, 5, 9, 16, LinesCfg<Rad<6, 5, 9>, 16>::THREADS, LinesCfg<Rad<6, 5, 9>, 16>::SMEM_BYTES, launch_lines_270_1},
    {270, 2, 9, 5, 6, 8, LinesCfg<Rad<9, 5, 6>, 8>::THREADS, LinesCfg<Rad<9, 5, 6>, 8>::SMEM_BYTES, launch_lines_270_2},
    {280, 0, 8, 5, 7, 16, LinesCfg<Rad<8, 5, 7>, 16>::THREADS, LinesCfg<Rad<8, 5, 7>, 16>::SMEM_BYTES, launch_lines_280_0},
    {280, 1, 7, 5, 8, 16, LinesCfg<Rad<7, 5, 8>, 16>::THREADS, LinesCfg<Rad<7, 5, 8>, 16>::SMEM_BYTES, launch_lines_280_1},
    {280, 2, 8, 5, 7, 8, LinesCfg<Rad<8, 5, 7>, 8>::THREADS, LinesCfg<Rad<8, 5, 7>, 8>::SMEM_BYTES, launch_lines_280_2},
    {288, 0, 8, 6, 6, 16, LinesCfg<Rad<8, 6, 6>, 16>::THREADS, LinesCfg<Rad<8, 6, 6>, 16>::SMEM_BYTES, launch_lines_288_0},
    {288, 1, 6, 6, 8, 16, LinesCfg<Rad<6, 6, 8>, 16>::THREADS, LinesCfg<Rad<6, 6, 8>, 16>::SMEM_BYTES, launch_lines_288_1},
    {288, 2, 8, 6, 6, 8, LinesCfg<Rad<8, 6, 6>, 8>::THREADS, LinesCfg<Rad<8, 6, 6>, 8>::SMEM_BYTES, launch_lines_288_2},
    {294, 0, 7, 6, 7, 16, LinesCfg<Rad<7, 6, 7>, 16>::THREADS, LinesCfg<Rad<7, 6, 7>, 16>::SMEM_BYTES, launch_lines_294_0},
    {294, 1, 6, 7, 7, 16, LinesCfg<Rad<6, 7, 7>, 16>::THREADS, LinesCfg<Rad<6, 7, 7>, 16>::SMEM_BYTES, launch_lines_294_1},
    {294, 2, 7, 6, 7, 8, LinesCfg<Rad<7, 6, 7>, 8>::THREADS, LinesCfg<Rad<7, 6, 7>, 8>::SMEM_BYTES, launch_lines_294_2},
    {300, 0, 10, 5, 6, 16, LinesCfg<Rad<10, 5, 6>, 16>::THREADS, LinesCfg<Rad<10, 5, 6>, 16>::SMEM_BYTES, launch_lines_300_0},
    {300, 1, 6, 5, 10, 16, LinesCfg<Rad<6, 5, 10>, 16>::THREADS, LinesCfg<Rad<6, 5, 10>, 16>::SMEM_BYTES, launch_lines_300_1},
    {300, 2, 10, 5, 6, 8, LinesCfg<Rad<10, 5, 6>, 8>::THREADS, LinesCfg<Rad<10, 5, 6>, 8>::SMEM_BYTES, launch_lines_300_2},
    {315, 0, 9, 5, 7, 16, LinesCfg<Rad<9, 5, 7>, 16>::THREADS, LinesCfg<Rad<9, 5, 7>, 16>::SMEM_BYTES, launch_lines_315_0},
    {315, 1, 7, 5, 9, 16, LinesCfg<Rad<7, 5, 9>, 16>::THREADS, LinesCfg<Rad<7, 5, 9>, 16>::SMEM_BYTES, launch_lines_315_1},
    {315, 2, 9, 5, 7, 8, LinesCfg<Rad<9, 5, 7>, 8>::THREADS, LinesCfg<Rad<9, 5, 7>, 8>::SMEM_BYTES, launch_lines_315_2},
    {320, 0, 8, 5, 8, 16, LinesCfg<Rad<8, 5, 8>, 16>::THREADS, LinesCfg<Rad<8, 5, 8>, 16>::SMEM_BYTES, launch_lines_320_0},
    {320, 1, 5, 8, 8, 16, LinesCfg<Rad<5, 8, 8>, 16>::THREADS, LinesCfg<Rad<5, 8, 8>, 16>::SMEM_BYTES, launch_lines_320_1},
    {320, 2, 8, 5, 8, 8, LinesCfg<Rad<8, 5, 8>, 8>::THREADS, LinesCfg<Rad<8, 5, 8>, 8>::SMEM_BYTES, launch_lines_320_2},
    {324, 0, 9, 6, 6, 16, LinesCfg<Rad<9, 6, 6>, 16>::THREADS, LinesCfg<Rad<9, 6, 6>, 16>::SMEM_BYTES, launch_lines_324_0},
    {324, 1, 6, 6, 9, 16, LinesCfg<Rad<6, 6, 9>, 16>::THREADS, LinesCfg<Rad<6, 6, 9>, 16>::SMEM_BYTES, launch_lines_324_1},
    {324, 2, 9, 6, 6, 8, LinesCfg<Rad<9, 6, 6>, 8>::THREADS, LinesCfg<Rad<9, 6, 6>, 8>::SMEM_BYTES, launch_lines_324_2},
    {336, 0, 8, 6, 7, 16, LinesCfg<Rad<8, 6, 7>, 16>::THREADS, LinesCfg<Rad<8, 6, 7>, 16>::SMEM_BYTES, launch_lines_336_0},
    {336, 1, 7, 6, 8, 16, LinesCfg<Rad<7, 6, 8>, 16>::THREADS, LinesCfg<Rad<7, 6, 8>, 16>::SMEM_BYTES, launch_lines_336_1},
    {336, 2, 8, 6, 7, 8, LinesCfg<Rad<8, 6, 7>, 8>::THREADS, LinesCfg<Rad<8, 6, 7>, 8>::SMEM_BYTES, launch_lines_336_2},
    {343, 0, 7, 7, 7, 16, LinesCfg<Rad<7, 7, 7>, 16>::THREADS, LinesCfg<Rad<7, 7, 7>, 16>::SMEM_BYTES, launch_lines_343_0},
    {343, 1, 7, 7, 7, 8, LinesCfg<Rad<7, 7, 7>, 8>::THREADS, LinesCfg<Rad<7, 7, 7>, 8>::SMEM_BYTES, launch_lines_343_1},
    {350, 0, 10, 5, 7, 8, LinesCfg<Rad<10, 5, 7>, 8>::THREADS, LinesCfg<Rad<10, 5, 7>, 8>::SMEM_BYTES, launch_lines_350_0},
    {350, 1, 7, 5, 10, 8, LinesCfg<Rad<7, 5, 10>, 8>::THREADS, LinesCfg<Rad<7, 5, 10>, 8>::SMEM_BYTES, launch_lines_350_1},
    {350, 2, 10, 5, 7, 4, LinesCfg<Rad<10, 5, 7>, 4>::THREADS, LinesCfg<Rad<10, 5, 7>, 4>::SMEM_BYTES, launch_lines_350_2},
    {360, 0, 10, 6, 6, 16, LinesCfg<Rad<10, 6, 6>, 16>::THREADS, LinesCfg<Rad<10, 6, 6>, 16>::SMEM_BYTES, launch_lines_360_0},
    {360, 1, 6, 6, 10, 16, LinesCfg<Rad<6, 6, 10>, 16>::THREADS, LinesCfg<Rad<6, 6, 10>, 16>::SMEM_BYTES, launch_lines_360_1},
    {360, 2, 10, 6, 6, 8, LinesCfg<Rad<10, 6, 6>, 8>::THREADS, LinesCfg<Rad<10, 6, 6>, 8>::SMEM_BYTES, launch_lines_360_2},
    {375, 0, 15, 5, 5, 8, LinesCfg<Rad<15, 5, 5>, 8>::THREADS, LinesCfg<Rad<15, 5, 5>, 8>::SMEM_BYTES, launch_lines_375_0},
    {375, 1, 5, 5, 15, 8, LinesCfg<Rad<5, 5, 15>, 8>::THREADS, LinesCfg<Rad<5, 5, 15>, 8>::SMEM_BYTES, launch_lines_375_1},
    {375, 2, 15, 5, 5, 4, LinesCfg<Rad<15, 5, 5>, 4>::THREADS, LinesCfg<Rad<15, 5, 5>, 4>::SMEM_BYTES, launch_lines_375_2},
    {378, 0, 9, 6, 7, 16, LinesCfg<Rad<9, 6, 7>, 16>::THREADS, LinesCfg<Rad<9, 6, 7>, 16>::SMEM_BYTES, launch_lines_378_0},
    {378, 1, 7, 6, 9, 16, LinesCfg<Rad<7, 6, 9>, 16>::THREADS, LinesCfg<Rad<7, 6, 9>, 16>::SMEM_BYTES, launch_lines_378_1},
    {378, 2, 9, 6, 7, 8, LinesCfg<Rad<9, 6, 7>, 8>::THREADS, LinesCfg<Rad<9, 6, 7>, 8>::SMEM_BYTES, launch_lines_378_2},
    {384, 0, 8, 6, 8, 16, LinesCfg<Rad<8, 6, 8>, 16>::THREADS, LinesCfg<Rad<8, 6, 8>, 16>::SMEM_BYTES, launch_lines_384_0},
    {384, 1, 6, 8, 8, 16, LinesCfg<Rad<6, 8, 8>, 16>::THREADS, LinesCfg<Rad<6, 8, 8>, 16>::SMEM_BYTES, launch_lines_384_1},
    {384, 2, 8, 6, 8, 8, LinesCfg<Rad<8, 6, 8>, 8>::THREADS, LinesCfg<Rad<8, 6, 8>, 8>::SMEM_BYTES, launch_lines_384_2},
    {392, 0, 8, 7, 7, 16, LinesCfg<Rad<8, 7, 7>, 16>::THREADS, LinesCfg<Rad<8, 7, 7>, 16>::SMEM_BYTES, launch_lines_392_0},
    {392, 1, 7, 7, 8, 16, LinesCfg<Rad<7, 7, 8>, 16>::THREADS, LinesCfg<Rad<7, 7, 8>, 16>::SMEM_BYTES, launch_lines_392_1},
    {392, 2, 8, 7, 7, 8, LinesCfg<Rad<8, 7, 7>, 8>::THREADS, LinesCfg<Rad<8, 7, 7>, 8>::SMEM_BYTES, launch_lines_392_2},
    {400, 0, 10, 5, 8, 8, LinesCfg<Rad<10, 5, 8>, 8>::THREADS, LinesCfg<Rad<10, 5, 8>, 8>::SMEM_BYTES, launch_lines_400_0},
    {400, 1, 8, 5, 10, 8, LinesCfg<Rad<8, 5, 10>, 8>::THREADS, LinesCfg<Rad<8, 5, 10>, 8>::SMEM_BYTES, launch_lines_400_1},
    {400, 2, 10, 5, 8, 4, LinesCfg<Rad<10, 5, 8>, 4>::THREADS, LinesCfg<Rad<10, 5, 8>, 4>::SMEM_BYTES, launch_lines_400_2},
    {405, 0, 9, 5, 9, 8, LinesCfg<Rad<9, 5, 9>, 8>::THREADS, LinesCfg<Rad<9, 5, 9>, 8>::SMEM_BYTES, launch_lines_405_0},
    {405, 1, 5, 9, 9, 8, LinesCfg<Rad<5, 9, 9>, 8>::THREADS, LinesCfg<Rad<5, 9, 9>, 8>::SMEM_BYTES, launch_lines_405_1},
    {405, 2, 9, 5, 9, 4, LinesCfg<Rad<9, 5, 9>, 4>::THREADS, LinesCfg<Rad<9, 5, 9>, 4>::SMEM_BYTES, launch_lines_405_2},
    {420, 0, 10, 6, 7, 8, LinesCfg<Rad<10, 6, 7>, 8>::THREADS, LinesCfg<Rad<10, 6, 7>, 8>::SMEM_BYTES, launch_lines_420_0},
    {420, 1, 7, 6, 10, 8, LinesCfg<Rad<7, 6, 10>, 8>::THREADS, LinesCfg<Rad<7, 6, 10>, 8>::SMEM_BYTES, launch_lines_420_1},
    {420, 2, 10, 6, 7, 4, LinesCfg<Rad<10, 6, 7>, 4>::THREADS, LinesCfg<Rad<10, 6, 7>, 4>::SMEM_BYTES, launch_lines_420_2},
    {432, 0, 9, 6, 8, 8, LinesCfg<Rad<9, 6, 8>, 8>::THREADS, LinesCfg<Rad<9, 6, 8>, 8>::SMEM_BYTES, launch_lines_432_0},
    {432, 1, 8, 6, 9, 8, LinesCfg<Rad<8, 6, 9>, 8>::THREADS, LinesCfg<Rad<8, 6, 9>, 8>::SMEM_BYTES, launch_lines_432_1},
    {432, 2, 9, 6, 8, 4, LinesCfg<Rad<9, 6, 8>, 4>::THREADS, LinesCfg<Rad<9, 6, 8>, 4>::SMEM_BYTES, launch_lines_432_2},
    {441, 0, 9, 7, 7, 16, LinesCfg<Rad<9, 7, 7>, 16>::THREADS, LinesCfg<Rad<9, 7, 7>, 16>::SMEM_BYTES, launch_lines_441_0},
    {441, 1, 7, 7, 9, 16, LinesCfg<Rad<7, 7, 9>, 16>::THREADS, LinesCfg<Rad<7, 7, 9>, 16>::SMEM_BYTES, launch_lines_441_1},
    {441, 2, 9, 7, 7, 8, LinesCfg<Rad<9, 7, 7>, 8>::THREADS, LinesCfg<Rad<9, 7, 7>, 8>::SMEM_BYTES, launch_lines_441_2},
    {448, 0, 8, 7, 8, 16, LinesCfg<Rad<8, 7, 8>, 16>::THREADS, LinesCfg<Rad<8, 7, 8>, 16>::SMEM_BYTES, launch_lines_448_0},
    {448, 1, 7, 8, 8, 16, LinesCfg<Rad<7, 8, 8>, 16>::THREADS, LinesCfg<Rad<7, 8, 8>, 16>::SMEM_BYTES, launch_lines_448_1},
    {448, 2, 8, 7, 8, 8, LinesCfg<Rad<8, 7, 8>, 8>::THREADS, LinesCfg<Rad<8, 7, 8>, 8>::SMEM_BYTES, launch_lines_448_2},
    {450, 0, 10, 5, 9, 8, LinesCfg<Rad<10, 5, 9>, 8>::THREADS, LinesCfg<Rad<10, 5, 9>, 8>::SMEM_BYTES, launch_lines_450_0},
    {450, 1, 9, 5, 10, 8, LinesCfg<Rad<9, 5, 10>, 8>::THREADS, LinesCfg<Rad<9, 5, 10>, 8>::SMEM_BYTES, launch_lines_450_1},
    {450, 2, 10, 5, 9, 4, LinesCfg<Rad<10, 5, 9>, 4>::THREADS, LinesCfg<Rad<10, 5, 9>, 4>::SMEM_BYTES, launch_lines_450_2},
    {480, 0, 10, 6, 8, 8, LinesCfg<Rad<10, 6, 8>, 8>::THREADS, LinesCfg<Rad<10, 6, 8>, 8>::SMEM_BYTES, launch_lines_480_0},
    {480, 1, 8, 6, 10, 8, LinesCfg<Rad<8, 6, 10>, 8>::THREADS, LinesCfg<Rad<8, 6, 10>, 8>::SMEM_BYTES, launch_lines_480_1},
    {480, 2, 10, 6, 8, 4, LinesCfg<Rad<10, 6, 8>, 4>::THREADS, LinesCfg<Rad<10, 6, 8>, 4>::SMEM_BYTES, launch_lines_480_2},
    {486, 0, 9, 6, 9, 8, LinesCfg<Rad<9, 6, 9>, 8>::THREADS, LinesCfg<Rad<9, 6, 9>, 8>::SMEM_BYTES, launch_lines_486_0},
    {486, 1, 6, 9, 9, 8, LinesCfg<Rad<6, 9, 9>, 8>::THREADS, LinesCfg<Rad<6, 9, 9>, 8>::SMEM_BYTES, launch_lines_486_1},
    {486, 2, 9, 6, 9, 4, LinesCfg<Rad<9, 6, 9>, 4>::THREADS, LinesCfg<Rad<9, 6, 9>, 4>::SMEM_BYTES, launch_lines_486_2},
    {490, 0, 10, 7, 7, 8, LinesCfg<Rad<10, 7, 7>, 8>::THREADS, LinesCfg<Rad<10, 7, 7>, 8>::SMEM_BYTES, launch_lines_490_0},
    {490, 1, 7, 7, 10, 8, LinesCfg<Rad<7, 7, 10>, 8>::THREADS, LinesCfg<Rad<7, 7, 10>, 8>::SMEM_BYTES, launch_lines_490_1},
    {490, 2, 10, 7, 7, 4, LinesCfg<Rad<10, 7, 7>, 4>::THREADS, LinesCfg<Rad<10, 7, 7>, 4>::SMEM_BYTES, launch_lines_490_2},
    {500, 0, 10, 5, 10, 8, LinesCfg<Rad<10, 5, 10>, 8>::THREADS, LinesCfg<Rad<10, 5, 10>, 8>::SMEM_BYTES, launch_lines_500_0},
    {500, 1, 5, 10, 10, 8, LinesCfg<Rad<5, 10, 10>, 8>::THREADS, LinesCfg<Rad<5, 10, 10>, 8>::SMEM_BYTES, launch_lines_500_1},
    {500, 2, 10, 5, 10, 4, LinesCfg<Rad<10, 5, 10>, 4>::THREADS, LinesCfg<Rad<10, 5, 10>, 4>::SMEM_BYTES, launch_lines_500_2},
    {504, 0, 9, 7, 8, 8, LinesCfg<Rad<9, 7, 8>, 8>::THREADS, LinesCfg<Rad<9, 7, 8>, 8>::SMEM_BYTES, launch_lines_504_0},
    {504, 1, 8, 7, 9, 8, LinesCfg<Rad<8, 7, 9>, 8>::THREADS, LinesCfg<Rad<8, 7, 9>, 8>::SMEM_BYTES, launch_lines_504_1},
    {504, 2, 9, 7, 8, 4, LinesCfg<Rad<9, 7, 8>, 4>::THREADS, LinesCfg<Rad<9, 7, 8>, 4>::SMEM_BYTES, launch_lines_504_2},
    {512, 0, 8, 8, 8, 16, LinesCfg<Rad<8, 8, 8>, 16>::THREADS, LinesCfg<Rad<8, 8, 8>, 16>::SMEM_BYTES, launch_lines_512_0},
    {512, 1, 16, 4, 8, 8, LinesCfg<Rad<16, 4, 8>, 8>::THREADS, LinesCfg<Rad<16, 4, 8>, 8>::SMEM_BYTES, launch_lines_512_1},
    {512, 2, 8, 8, 8, 8, LinesCfg<Rad<8, 8, 8>, 8>::THREADS, LinesCfg<Rad<8, 8, 8>, 8>::SMEM_BYTES, launch_lines_512_2},
    {525, 0, 15, 5, 7, 8, LinesCfg<Rad<15, 5, 7>, 8>::THREADS, LinesCfg<Rad<15, 5, 7>, 8>::SMEM_BYTES, launch_lines_525_0},
    {525, 1, 7, 5, 15, 8, LinesCfg<Rad<7, 5, 15>, 8>::THREADS, LinesCfg<Rad<7, 5, 15>, 8>::SMEM_BYTES, launch_lines_525_1},
    {525, 2, 15, 5, 7, 4, LinesCfg<Rad<15, 5, 7>, 4>::THREADS, LinesCfg<Rad<15, 5, 7>, 4>::SMEM_BYTES, launch_lines_525_2},
    {540, 0, 10, 6, 9, 8, LinesCfg<Rad<10, 6, 9>, 8>::THREADS, LinesCfg<Rad<10, 6, 9>, 8>::SMEM_BYTES, launch_lines_540_0},
    {540, 1, 9, 6, 10, 8, LinesCfg<Rad<9, 6, 10>, 8>::THREADS, LinesCfg<Rad<9, 6, 10>, 8>::SMEM_BYTES, launch_lines_540_1},
    {540, 2, 10, 6, 9, 4, LinesCfg<Rad<10, 6, 9>, 4>::THREADS, LinesCfg<Rad<10, 6, 9>, 4>::SMEM_BYTES, launch_lines_540_2},
    {560, 0, 10, 7, 8, 8, LinesCfg<Rad<10, 7, 8>, 8>::THREADS, LinesCfg<Rad<10, 7, 8>, 8>::SMEM_BYTES, launch_lines_560_0},
    {560, 1, 8, 7, 10, 8, LinesCfg<Rad<8, 7, 10>, 8>::THREADS, LinesCfg<Rad<8, 7, 10>, 8>::SMEM_BYTES, launch_lines_560_1},
    {560, 2, 10, 7, 8, 4, LinesCfg<Rad<10, 7, 8>, 4>::THREADS, LinesCfg<Rad<10, 7, 8>, 4>::SMEM_BYTES, launch_lines_560_2},
    {567, 0, 9, 7, 9, 8, LinesCfg<Rad<9, 7, 9>, 8>::THREADS, LinesCfg<Rad<9, 7, 9>, 8>::SMEM_BYTES, launch_lines_567_0},
    {567, 1, 7, 9, 9, 8, LinesCfg<Rad<7, 9, 9>, 8>::THREADS, LinesCfg<Rad<7, 9, 9>, 8>::SMEM_BYTES, launch_lines_567_1},
    {567, 2, 9, 7, 9, 4, LinesCfg<Rad<9, 7, 9>, 4>::THREADS, LinesCfg<Rad<9, 7, 9>, 4>::SMEM_BYTES, launch_lines_567_2},
    {576, 0, 9, 8, 8, 8, LinesCfg<Rad<9, 8, 8>, 8>::THREADS, LinesCfg<Rad<9, 8, 8>, 8>::SMEM_BYTES, launch_lines_576_0},
    {576, 1, 8, 8, 9, 8, LinesCfg<Rad<8, 8, 9>, 8>::THREADS, LinesCfg<Rad<8, 8, 9>, 8>::SMEM_BYTES, launch_lines_576_1},
    {576, 2, 9, 8, 8, 4, LinesCfg<Rad<9, 8, 8>, 4>::THREADS, LinesCfg<Rad<9, 8, 8>, 4>::SMEM_BYTES, launch_lines_576_2},
    {588, 0, 12, 7, 7, 8, LinesCfg<Rad<12, 7, 7>, 8>::THREADS, LinesCfg<Rad<12, 7, 7>, 8>::SMEM_BYTES, launch_lines_588_0},
    {588, 1, 7, 7, 12, 8, LinesCfg<Rad<7, 7, 12>, 8>::THREADS, LinesCfg<Rad<7, 7, 12>, 8>::SMEM_BYTES, launch_lines_588_1},
    {588, 2, 12, 7, 7, 4, LinesCfg<Rad<12, 7, 7>, 4>::THREADS, LinesCfg<Rad<12, 7, 7>, 4>::SMEM_BYTES, launch_lines_588_2},
    {600, 0, 10, 6, 10, 8, LinesCfg<Rad<10, 6, 10>, 8>::THREADS, LinesCfg<Rad<10, 6, 10>, 8>::SMEM_BYTES, launch_lines_600_0},
    {600, 1, 6, 10, 10, 8, LinesCfg<Rad<6, 10, 10>, 8>::THREADS, LinesCfg<Rad<6, 10, 10>, 8>::SMEM_BYTES, launch_lines_600_1},
    {600, 2, 10, 6, 10, 4, LinesCfg<Rad<10, 6, 10>, 4>::THREADS, LinesCfg<Rad<10, 6, 10>, 4>::SMEM_BYTES, launch_lines_600_2},
    {630, 0, 10, 7, 9, 8, LinesCfg<Rad<10, 7, 9>, 8>::THREADS, LinesCfg<Rad<10, 7, 9>, 8>::SMEM_BYTES, launch_lines_630_0},
    {630, 1, 9, 7, 10, 8, LinesCfg<Rad<9, 7, 10>, 8>::THREADS, LinesCfg<Rad<9, 7, 10>, 8>::SMEM_BYTES, launch_lines_630_1},
    {630, 2, 10, 7, 9, 4, LinesCfg<Rad<10, 7, 9>, 4>::THREADS, LinesCfg<Rad<10, 7, 9>, 4>::SMEM_BYTES, launch_lines_630_2},
    {640, 0, 10, 8, 8, 8, LinesCfg<Rad<10, 8, 8>, 8>::THREADS, LinesCfg<Rad<10, 8, 8>, 8>::SMEM_BYTES, launch_lines_640_0},
    {640, 1, 8, 8, 10, 8, LinesCfg<Rad<8, 8, 10>, 8>::THREADS, LinesCfg<Rad<8, 8, 10>, 8>::SMEM_BYTES, launch_lines_640_1},
    {640, 2, 10, 8, 8, 4, LinesCfg<Rad<10, 8, 8>, 4>::THREADS, LinesCfg<Rad<10, 8, 8>, 4>::SMEM_BYTES, launch_lines_640_2},
    {648, 0, 9, 8, 9, 8, LinesCfg<Rad<9, 8, 9>, 8>::THREADS, LinesCfg<Rad<9, 8, 9>, 8>::SMEM_BYTES, launch_lines_648_0},
    {648, 1, 8, 9, 9, 8, LinesCfg<Rad<8, 9, 9>, 8>::THREADS, LinesCfg<Rad<8, 9, 9>, 8>::SMEM_BYTES, launch_lines_648_1},
    {648, 2, 9, 8, 9, 4, LinesCfg<Rad<9, 8, 9>, 4>::THREADS, LinesCfg<Rad<9, 8, 9>, 4>::SMEM_BYTES, launch_lines_648_2},
    {672, 0, 12, 7, 8, 8, LinesCfg<Rad<12, 7, 8>, 8>::THREADS, LinesCfg<Rad<12, 7, 8>, 8>::SMEM_BYTES, launch_lines_672_0},
    {672, 1, 8, 7, 12, 8, LinesCfg<Rad<8, 7, 12>, 8>::THREADS, LinesCfg<Rad<8, 7, 12>, 8>::SMEM_BYTES, launch_lines_672_1},
    {672, 2, 12, 7, 8, 4, LinesCfg<Rad<12, 7, 8>, 4>::THREADS, LinesCfg<Rad<12, 7, 8>, 4>::SMEM_BYTES, launch_lines_672_2},
    {675, 0, 15, 5, 9, 4, LinesCfg<Rad<15, 5, 9>, 4>::THREADS, LinesCfg<Rad<15, 5, 9>, 4>::SMEM_BYTES, launch_lines_675_0},
    {675, 1, 9, 5, 15, 4, LinesCfg<Rad<9, 5, 15>, 4>::THREADS, LinesCfg<Rad<9, 5, 15>, 4>::SMEM_BYTES, launch_lines_675_1},
    {675, 2, 15, 5, 9, 2, LinesCfg<Rad<15, 5, 9>, 2>::THREADS, LinesCfg<Rad<15, 5, 9>, 2>::SMEM_BYTES, launch_lines_675_2},
    {686, 0, 14, 7, 7, 8, LinesCfg<Rad<14, 7, 7>, 8>::THREADS, LinesCfg<Rad<14, 7, 7>, 8>::SMEM_BYTES, launch_lines_686_0},
    {686, 1, 7, 7, 14, 8, LinesCfg<Rad<7, 7, 14>, 8>::THREADS, LinesCfg<Rad<7, 7, 14>, 8>::SMEM_BYTES, launch_lines_686_1},
    {686, 2, 14, 7, 7, 4, LinesCfg<Rad<14, 7, 7>, 4>::THREADS, LinesCfg<Rad<14, 7, 7>, 4>::SMEM_BYTES, launch_lines_686_2},
    {700, 0, 10, 7, 10, 8, LinesCfg<Rad<10, 7, 10>, 8>::THREADS, LinesCfg<Rad<10, 7, 10>, 8>::SMEM_BYTES, launch_lines_700_0},
    {700, 1, 7, 10, 10, 8, LinesCfg<Rad<7, 10, 10>, 8>::THREADS, LinesCfg<Rad<7, 10, 10>, 8>::SMEM_BYTES, launch_lines_700_1},
    {700, 2, 10, 7, 10, 4, LinesCfg<Rad<10, 7, 10>, 4>::THREADS, LinesCfg<Rad<10, 7, 10>, 4>::SMEM_BYTES, launch_lines_700_2},
    {720, 0, 10, 8, 9, 8, LinesCfg<Rad<10, 8, 9>, 8>::THREADS, LinesCfg<Rad<10, 8, 9>, 8>::SMEM_BYTES, launch_lines_720_0},
    {720, 1, 9, 8, 10, 8, LinesCfg<Rad<9, 8, 10>, 8>::THREADS, LinesCfg<Rad<9, 8, 10>, 8>::SMEM_BYTES, launch_lines_720_1},
    {720, 2, 10, 8, 9, 4, LinesCfg<Rad<10, 8, 9>, 4>::THREADS, LinesCfg<Rad<10, 8, 9>, 4>::SMEM_BYTES, launch_lines_720_2},
    {729, 0, 9, 9, 9, 8, LinesCfg<Rad<9, 9, 9>, 8>::THREADS, LinesCfg<Rad<9, 9, 9>, 8>::SMEM_BYTES, launch_lines_729_0},
    {729, 1, 9, 9, 9, 4, LinesCfg<Rad<9, 9, 9>, 4>::THREADS, LinesCfg<Rad<9, 9, 9>, 4>::SMEM_BYTES, launch_lines_729_1},
    {735, 0, 15, 7, 7, 8, LinesCfg<Rad<15, 7, 7>, 8>::THREADS, LinesCfg<Rad<15, 7, 7>, 8>::SMEM_BYTES, launch_lines_735_0},
    {735, 1, 7, 7, 15, 8, LinesCfg<Rad<7, 7, 15>, 8>::THREADS, LinesCfg<Rad<7, 7, 15>, 8>::SMEM_BYTES, launch_lines_735_1},
    {735, 2, 15, 7, 7, 4, LinesCfg<Rad<15, 7, 7>, 4>::THREADS, LinesCfg<Rad<15, 7, 7>, 4>::SMEM_BYTES, launch_lines_735_2},
    {750, 0, 15, 5, 10, 4, LinesCfg<Rad<15, 5, 10>, 4>::THREADS, LinesCfg<Rad<15, 5, 10>, 4>::SMEM_BYTES, launch_lines_750_0},
    {750, 1, 10, 5, 15, 4, LinesCfg<Rad<10, 5, 15>, 4>::THREADS, LinesCfg<Rad<10, 5, 15>, 4>::SMEM_BYTES, launch_lines_750_1},
    {750, 2, 15, 5, 10, 2, LinesCfg<Rad<15, 5, 10>, 2>::THREADS, LinesCfg<Rad<15, 5, 10>, 2>::SMEM_BYTES, launch_lines_750_2},
    {756, 0, 12, 7, 9, 8, LinesCfg<Rad<12, 7, 9>, 8>::THREADS, LinesCfg<Rad<12, 7, 9>, 8>::SMEM_BYTES, launch_lines_756_0},
    {756, 1, 9, 7, 12, 8, LinesCfg<Rad<9, 7, 12>, 8>::THREADS, LinesCfg<Rad<9, 7, 12>, 8>::SMEM_BYTES, launch_lines_756_1},
    {756, 2, 12, 7, 9, 4, LinesCfg<Rad<12, 7, 9>, 4>::THREADS, LinesCfg<Rad<12, 7, 9>, 4>::SMEM_BYTES, launch_lines_756_2},
    {768, 0, 12, 8, 8, 8, LinesCfg<Rad<12, 8, 8>, 8>::THREADS, LinesCfg<Rad<12, 8, 8>, 8>::SMEM_BYTES, launch_lines_768_0},
    {768, 1, 8, 8, 12, 8, LinesCfg<Rad<8, 8, 12>, 8>::THREADS, LinesCfg<Rad<8, 8, 12>, 8>::SMEM_BYTES, launch_lines_768_1},
    {768, 2, 12, 8, 8, 4, LinesCfg<Rad<12, 8, 8>, 4>::THREADS, LinesCfg<Rad<12, 8, 8>, 4>::SMEM_BYTES, launch_lines_768_2},
    {784, 0, 14, 7, 8, 8, LinesCfg<Rad<14, 7, 8>, 8>::THREADS, LinesCfg<Rad<14, 7, 8>, 8>::SMEM_BYTES, launch_lines_784_0},
    {784, 1, 8, 7, 14, 8, LinesCfg<Rad<8, 7, 14>, 8>::THREADS, LinesCfg<Rad<8, 7, 14>, 8>::SMEM_BYTES, launch_lines_784_1},
    {784, 2, 14, 7, 8, 4, LinesCfg<Rad<14, 7, 8>, 4>::THREADS, LinesCfg<Rad<14, 7, 8>, 4>::SMEM_BYTES, launch_lines_784_2},
    {800, 0, 10, 8, 10, 8, LinesCfg<Rad<10, 8, 10>, 8>::THREADS, LinesCfg<Rad<10, 8, 10>, 8>::SMEM_BYTES, launch_lines_800_0},
    {800, 1, 8, 10, 10, 8, LinesCfg<Rad<8, 10, 10>, 8>::THREADS, LinesCfg<Rad<8, 10, 10>, 8>::SMEM_BYTES, launch_lines_800_1},
    {800, 2, 10, 8, 10, 4, LinesCfg<Rad<10, 8, 10>, 4>::THREADS, LinesCfg<Rad<10, 8, 10>, 4>::SMEM_BYTES, launch_lines_800_2},
    {810, 0, 10, 9, 9, 8, LinesCfg<Rad<10, 9, 9>, 8>::THREADS, LinesCfg<Rad<10, 9, 9>, 8>::SMEM_BYTES, launch_lines_810_0},
    {810, 1, 9, 9, 10, 8, LinesCfg<Rad<9, 9, 10>, 8>::THREADS, LinesCfg<Rad<9, 9, 10>, 8>::SMEM_BYTES, launch_lines_810_1},
    {810, 2, 10, 9, 9, 4, LinesCfg<Rad<10, 9, 9>, 4>::THREADS, LinesCfg<Rad<10, 9, 9>, 4>::SMEM_BYTES, launch_lines_810_2},
    {840, 0, 12, 7, 10, 8, LinesCfg<Rad<12, 7, 10>, 8>::THREADS, LinesCfg<Rad<12, 7, 10>, 8>::SMEM_BYTES, launch_lines_840_0},
    {840, 1, 10, 7, 12, 8, LinesCfg<Rad<10, 7, 12>, 8>::THREADS, LinesCfg<Rad<10, 7, 12>, 8>::SMEM_BYTES, launch_lines_840_1},
    {840, 2, 12, 7, 10, 4, LinesCfg<Rad<12, 7, 10>, 4>::THREADS, LinesCfg<Rad<12, 7, 10>, 4>::SMEM_BYTES, launch_lines_840_2},
    {864, 0, 12, 8, 9, 8, LinesCfg<Rad<12, 8, 9>, 8>::THREADS, LinesCfg<Rad<12, 8, 9>, 8>::SMEM_BYTES, launch_lines_864_0},
    {864, 1, 9, 8, 12, 8, LinesCfg<Rad<9, 8, 12>, 8>::THREADS, LinesCfg<Rad<9, 8, 12>, 8>::SMEM_BYTES, launch_lines_864_1},
    {864, 2, 12, 8, 9, 4, LinesCfg<Rad<12, 8, 9>, 4>::THREADS, LinesCfg<Rad<12, 8, 9>, 4>::SMEM_BYTES, launch_lines_864_2},
    {882, 0, 14, 7, 9, 8, LinesCfg<Rad<14, 7, 9>, 8>::THREADS, LinesCfg<Rad<14, 7, 9>, 8>::SMEM_BYTES, launch_lines_882_0},
    {882, 1, 9, 7, 14, 8, LinesCfg<Rad<9, 7, 14>, 8>::THREADS, LinesCfg<Rad<9, 7, 14>, 8>::SMEM_BYTES, launch_lines_882_1},
    {882, 2, 14, 7, 9, 4, LinesCfg<Rad<14, 7, 9>, 4>::THREADS, LinesCfg<Rad<14, 7, 9>, 4>::SMEM_BYTES, launch_lines_882_2},
    {896, 0, 14, 8, 8, 8, LinesCfg<Rad<14, 8, 8>, 8>::THREADS, LinesCfg<Rad<14, 8, 8>, 8>::SMEM_BYTES, launch_lines_896_0},
    {896, 1, 8, 8, 14, 8, LinesCfg<Rad<8, 8, 14>, 8>::THREADS, LinesCfg<Rad<8, 8, 14>, 8>::SMEM_BYTES, launch_lines_896_1},
    {896, 2, 14, 8, 8, 4, LinesCfg<Rad<14, 8, 8>, 4>::THREADS, LinesCfg<Rad<14, 8, 8>, 4>::SMEM_BYTES, launch_lines_896_2},
    {900, 0, 10, 9, 10, 8, LinesCfg<Rad<10, 9, 10>, 8>::THREADS, LinesCfg<Rad<10, 9, 10>, 8>::SMEM_BYTES, launch_lines_900_0},
    {900, 1, 9, 10, 10, 8, LinesCfg<Rad<9, 10, 10>, 8>::THREADS, LinesCfg<Rad<9, 10, 10>, 8>::SMEM_BYTES, launch_lines_900_1},
    {900, 2, 10, 9, 10, 4, LinesCfg<Rad<10, 9, 10>, 4>::THREADS, LinesCfg<Rad<10, 9, 10>, 4>::SMEM_BYTES, launch_lines_900_2},
    {945, 0, 15, 7, 9, 4, LinesCfg<Rad<15, 7, 9>, 4>::THREADS, LinesCfg<Rad<15, 7, 9>, 4>::SMEM_BYTES, launch_lines_945_0},
    {945, 1, 9, 7, 15, 4, LinesCfg<Rad<9, 7, 15>, 4>::THREADS, LinesCfg<Rad<9, 7, 15>, 4>::SMEM_BYTES, launch_lines_945_1},
    {945, 2, 15, 7, 9, 2, LinesCfg<Rad<15, 7, 9>, 2>::THREADS, LinesCfg<Rad<15, 7, 9>, 2>::SMEM_BYTES, launch_lines_945_2},
    {960, 0, 12, 8, 10, 8, LinesCfg<Rad<12, 8, 10>, 8>::THREADS, LinesCfg<Rad<12, 8, 10>, 8>::SMEM_BYTES, launch_lines_960_0},
    {960, 1, 10, 8, 12, 8, LinesCfg<Rad<10, 8, 12>, 8>::THREADS, LinesCfg<Rad<10, 8, 12>, 8>::SMEM_BYTES, launch_lines_960_1},
    {960, 2, 12, 8, 10, 4, LinesCfg<Rad<12, 8, 10>, 4>::THREADS, LinesCfg<Rad<12, 8, 10>, 4>::SMEM_BYTES, launch_lines_960_2},
    {972, 0, 12, 9, 9, 8, LinesCfg<Rad<12, 9, 9>, 8>::THREADS, LinesCfg<Rad<12, 9, 9>, 8>::SMEM_BYTES, launch_lines_972_0},
    {972, 1, 9, 9, 12, 8, LinesCfg<Rad<9, 9, 12>, 8>::THREADS, LinesCfg<Rad<9, 9, 12>, 8>::SMEM_BYTES, launch_lines_972_1},
    {972, 2, 12, 9, 9, 4, LinesCfg<Rad<12, 9, 9>, 4>::THREADS, LinesCfg<Rad<12, 9, 9>, 4>::SMEM_BYTES, launch_lines_972_2},
    {980, 0, 14, 7, 10, 4, LinesCfg<Rad<14, 7, 10>, 4>::THREADS, LinesCfg<Rad<14, 7, 10>, 4>::SMEM_BYTES, launch_lines_980_0},
    {980, 1, 10, 7, 14, 4, LinesCfg<Rad<10, 7, 14>, 4>::THREADS, LinesCfg<Rad<10, 7, 14>, 4>::SMEM_BYTES, launch_lines_980_1},
    {980, 2, 14, 7, 10, 2, LinesCfg<Rad<14, 7, 10>, 2>::THREADS, LinesCfg<Rad<14, 7, 10>, 2>::SMEM_BYTES, launch_lines_980_2},
    {1000, 0, 10, 10, 10, 8, LinesCfg<Rad<10, 10, 10>, 8>::THREADS, LinesCfg<Rad<10, 10, 10>, 8>::SMEM_BYTES, launch_lines_1000_0},
    {1000, 1, 10, 10, 10, 4, LinesCfg<Rad<10, 10, 10>, 4>::THREADS, LinesCfg<Rad<10, 10, 10>, 4>::SMEM_BYTES, launch_lines_1000_1},
    {1008, 0, 14, 8, 9, 8, LinesCfg<Rad<14, 8, 9>, 8>::THREADS, LinesCfg<Rad<14, 8, 9>, 8>::SMEM_BYTES, launch_lines_1008_0},
    {1008, 1, 9, 8, 14, 8, LinesCfg<Rad<9, 8, 14>, 8>::THREADS, LinesCfg<Rad<9, 8, 14>, 8>::SMEM_BYTES, launch_lines_1008_1},
    {1008, 2, 14, 8, 9, 4, LinesCfg<Rad<14, 8, 9>, 4>::THREADS, LinesCfg<Rad<14, 8, 9>, 4>::SMEM_BYTES, launch_lines_1008_2},
    {1024, 0, 16, 8, 8, 8, LinesCfg<Rad<16, 8, 8>, 8>::THREADS, LinesCfg<Rad<16, 8, 8>, 8>::SMEM_BYTES, launch_lines_1024_0},
    {1024, 1, 8, 8, 16, 8, LinesCfg<Rad<8, 8, 16>, 8>::THREADS, LinesCfg<Rad<8, 8, 16>, 8>::SMEM_BYTES, launch_lines_1024_1},
    {1024, 2, 16, 8, 8, 4, LinesCfg<Rad<16, 8, 8>, 4>::THREADS, LinesCfg<Rad<16, 8, 8>, 4>::SMEM_BYTES, launch_lines_1024_2},
    {1050, 0, 15, 7, 10, 4, LinesCfg<Rad<15, 7, 10>, 4>::THREADS, LinesCfg<Rad<15, 7, 10>, 4>::SMEM_BYTES, launch_lines_1050_0},
    {1050, 1, 10, 7, 15, 4, LinesCfg<Rad<10, 7, 15>, 4>::THREADS, LinesCfg<Rad<10, 7, 15>, 4>::SMEM_BYTES, launch_lines_1050_1},
    {1050, 2, 15, 7, 10, 2, LinesCfg<Rad<15, 7, 10>, 2>::THREADS, LinesCfg<Rad<15, 7, 10>, 2>::SMEM_BYTES, launch_lines_1050_2},
    {1080, 0, 12, 9, 10, 8, LinesCfg<Rad<12, 9, 10>, 8>::THREADS, LinesCfg<Rad<12, 9, 10>, 8>::SMEM_BYTES, launch_lines_1080_0},
    {1080, 1, 10, 9, 12, 8, LinesCfg<Rad<10, 9, 12>, 8>::THREADS, LinesCfg<Rad<10, 9, 12>, 8>::SMEM_BYTES, launch_lines_1080_1},
    {1080, 2, 12, 9, 10, 4, LinesCfg<Rad<12, 9, 10>, 4>::THREADS, LinesCfg<Rad<12, 9, 10>, 4>::SMEM_BYTES, launch_lines_1080_2},
    {1120, 0, 14, 8, 10, 4, LinesCfg<Rad<14, 8, 10>, 4>::THREADS, LinesCfg<Rad<14, 8, 10>, 4>::SMEM_BYTES, launch_lines_1120_0},
    {1120, 1, 10, 8, 14, 4, LinesCfg<Rad<10, 8, 14>, 4>::THREADS, LinesCfg<Rad<10, 8, 14>, 4>::SMEM_BYTES, launch_lines_1120_1},
    {1120, 2, 14, 8, 10, 2, LinesCfg<Rad<14, 8, 10>, 2>::THREADS, LinesCfg<Rad<14, 8, 10>, 2>::SMEM_BYTES, launch_lines_1120_2},
    {1125, 0, 15, 5, 15, 4, LinesCfg<Rad<15, 5, 15>, 4>::THREADS, LinesCfg<Rad<15, 5, 15>, 4>::SMEM_BYTES, launch_lines_1125_0},
    {1125, 1, 5, 15, 15, 4, LinesCfg<Rad<5, 15, 15>, 4>::THREADS, LinesCfg<Rad<5, 15, 15>, 4>::SMEM_BYTES, launch_lines_1125_1},
    {1125, 2, 15, 5, 15, 2, LinesCfg<Rad<15, 5, 15>, 2>::THREADS, LinesCfg<Rad<15, 5, 15>, 2>::SMEM_BYTES, launch_lines_1125_2},
    {1134, 0, 14, 9, 9, 8, LinesCfg<Rad<14, 9, 9>, 8>::THREADS, LinesCfg<Rad<14, 9, 9>, 8>::SMEM_BYTES, launch_lines_1134_0},
    {1134, 1, 9, 9, 14, 8, LinesCfg<Rad<9, 9, 14>, 8>::THREADS, LinesCfg<Rad<9, 9, 14>, 8>::SMEM_BYTES, launch_lines_1134_1},
    {1134, 2, 14, 9, 9, 4, LinesCfg<Rad<14, 9, 9>, 4>::THREADS, LinesCfg<Rad<14, 9, 9>, 4>::SMEM_BYTES, launch_lines_1134_2},
    {1152, 0, 12, 8, 12, 4, LinesCfg<Rad<12, 8, 12>, 4>::THREADS, LinesCfg<Rad<12, 8, 12>, 4>::SMEM_BYTES, launch_lines_1152_0},
    {1152, 1, 8, 12, 12, 4, LinesCfg<Rad<8, 12, 12>, 4>::THREADS, LinesCfg<Rad<8, 12, 12>, 4>::SMEM_BYTES, launch_lines_1152_1},
    {1152, 2, 12, 8, 12, 2, LinesCfg<Rad<12, 8, 12>, 2>::THREADS, LinesCfg<Rad<12, 8, 12>, 2>::SMEM_BYTES, launch_lines_1152_2},
    {1176, 0, 14, 7, 12, 4, LinesCfg<Rad<14, 7, 12>, 4>::THREADS, LinesCfg<Rad<14, 7, 12>, 4>::SMEM_BYTES, launch_lines_1176_0},
    {1176, 1, 12, 7, 14, 4, LinesCfg<Rad<12, 7, 14>, 4>::THREADS, LinesCfg<Rad<12, 7, 14>, 4>::SMEM_BYTES, launch_lines_1176_1},
    {1176, 2, 14, 7, 12, 2, LinesCfg<Rad<14, 7, 12>, 2>::THREADS, LinesCfg<Rad<14, 7, 12>, 2>::SMEM_BYTES, launch_lines_1176_2},
    {1200, 0, 12, 10, 10, 8, LinesCfg<Rad<12, 10, 10>, 8>::THREADS, LinesCfg<Rad<12, 10, 10>, 8>::SMEM_BYTES, launch_lines_1200_0},
    {1200, 1, 10, 10, 12, 8, LinesCfg<Rad<10, 10, 12>, 8>::THREADS, LinesCfg<Rad<10, 10, 12>, 8>::SMEM_BYTES, launch_lines_1200_1},
    {1200, 2, 12, 10, 10, 4, LinesCfg<Rad<12, 10, 10>, 4>::THREADS, LinesCfg<Rad<12, 10, 10>, 4>::SMEM_BYTES, launch_lines_1200_2},
    {1215, 0, 15, 9, 9, 4, LinesCfg<Rad<15, 9, 9>, 4>::THREADS, LinesCfg<Rad<15, 9, 9>, 4>::SMEM_BYTES, launch_lines_1215_0},
    {1215, 1, 9, 9, 15, 4, LinesCfg<Rad<9, 9, 15>, 4>::THREADS, LinesCfg<Rad<9, 9, 15>, 4>::SMEM_BYTES, launch_lines_1215_1},
    {1215, 2, 15, 9, 9, 2, LinesCfg<Rad<15, 9, 9>, 2>::THREADS, LinesCfg<Rad<15, 9, 9>, 2>::SMEM_BYTES, launch_lines_1215_2},
    {1260, 0, 14, 9, 10, 4, LinesCfg<Rad<14, 9, 10>, 4>::THREADS, LinesCfg<Rad<14, 9, 10>, 4>::SMEM_BYTES, launch_lines_1260_0},
    {1260, 1, 10, 9, 14, 4, LinesCfg<Rad<10, 9, 14>, 4>::THREADS, LinesCfg<Rad<10, 9, 14>, 4>::SMEM_BYTES, launch_lines_1260_1},
    {1260, 2, 14, 9, 10, 2, LinesCfg<Rad<14, 9, 10>, 2>::THREADS, LinesCfg<Rad<14, 9, 10>, 2>::SMEM_BYTES, launch_lines_1260_2},
    {1280, 0, 16, 8, 10, 4, LinesCfg<Rad<16, 8, 10>, 4>::THREADS, LinesCfg<Rad<16, 8, 10>, 4>::SMEM_BYTES, launch_lines_1280_0},
    {1280, 1, 10, 8, 16, 4, LinesCfg<Rad<10, 8, 16>, 4>::THREADS, LinesCfg<Rad<10, 8, 16>, 4>::SMEM_BYTES, launch_lines_1280_1},
    {1280, 2, 16, 8, 10, 2, LinesCfg<Rad<16, 8, 10>, 2>::THREADS, LinesCfg<Rad<16, 8, 10>, 2>::SMEM_BYTES, launch_lines_1280_2},
    {1296, 0, 12, 9, 12, 4, LinesCfg<Rad<12, 9, 12>, 4>::THREADS, LinesCfg<Rad<12, 9, 12>, 4>::SMEM_BYTES, launch_lines_1296_0},
    {1296, 1, 9, 12, 12, 4, LinesCfg<Rad<9, 12, 12>, 4>::THREADS, LinesCfg<Rad<9, 12, 12>, 4>::SMEM_BYTES, launch_lines_1296_1},
    {1296, 2, 12, 9, 12, 2, LinesCfg<Rad<12, 9, 12>, 2>::THREADS, LinesCfg<Rad<12, 9, 12>, 2>::SMEM_BYTES, launch_lines_1296_2},
    {1344, 0, 14, 8, 12, 4, LinesCfg<Rad<14, 8, 12>, 4>::THREADS, LinesCfg<Rad<14, 8, 12>, 4>::SMEM_BYTES, launch_lines_1344_0},
    {1344, 1, 12, 8, 14, 4, LinesCfg<Rad<12, 8, 14>, 4>::THREADS, LinesCfg<Rad<12, 8, 14>, 4>::SMEM_BYTES, launch_lines_1344_1},
    {1344, 2, 14, 8, 12, 2, LinesCfg<Rad<14, 8, 12>, 2>::THREADS, LinesCfg<Rad<14, 8, 12>, 2>::SMEM_BYTES, launch_lines_1344_2},
    {1350, 0, 15, 9, 10, 4, LinesCfg<Rad<15, 9, 10>, 4>::THREADS, LinesCfg<Rad<15, 9, 10>, 4>::SMEM_BYTES, launch_lines_1350_0},
    {1350, 1, 10, 9, 15, 4, LinesCfg<Rad<10, 9, 15>, 4>::THREADS, LinesCfg<Rad<10, 9, 15>, 4>::SMEM_BYTES, launch_lines_1350_1},
    {1350, 2, 15, 9, 10, 2, LinesCfg<Rad<15, 9, 10>, 2>::THREADS, LinesCfg<Rad<15, 9, 10>, 2>::SMEM_BYTES, launch_lines_1350_2},
    {1372, 0, 14, 7, 14, 4, LinesCfg<Rad<14, 7, 14>, 4>::THREADS, LinesCfg<Rad<14, 7, 14>, 4>::SMEM_BYTES, launch_lines_1372_0},
    {1372, 1, 7, 14, 14, 4, LinesCfg<Rad<7, 14, 14>, 4>::THREADS, LinesCfg<Rad<7, 14, 14>, 4>::SMEM_BYTES, launch_lines_1372_1},
    {1372, 2, 14, 7, 14, 2, LinesCfg<Rad<14, 7, 14>, 2>::THREADS, LinesCfg<Rad<14, 7, 14>, 2>::SMEM_BYTES, launch_lines_1372_2},
    {1400, 0, 14, 10, 10, 4, LinesCfg<Rad<14, 10, 10>, 4>::THREADS, LinesCfg<Rad<14, 10, 10>, 4>::SMEM_BYTES, launch_lines_1400_0},
    {1400, 1, 10, 10, 14, 4, LinesCfg<Rad<10, 10, 14>, 4>::THREADS, LinesCfg<Rad<10, 10, 14>, 4>::SMEM_BYTES, launch_lines_1400_1},
    {1400, 2, 14, 10, 10, 2, LinesCfg<Rad<14, 10, 10>, 2>::THREADS, LinesCfg<Rad<14, 10, 10>, 2>::SMEM_BYTES, launch_lines_1400_2},
    {1440, 0, 12, 10, 12, 4, LinesCfg<Rad<12, 10, 12>, 4>::THREADS, LinesCfg<Rad<12, 10, 12>, 4>::SMEM_BYTES, launch_lines_1440_0},
    {1440, 1, 10, 12, 12, 4, LinesCfg<Rad<10, 12, 12>, 4>::THREADS, LinesCfg<Rad<10, 12, 12>, 4>::SMEM_BYTES, launch_lines_1440_1},
    {1440, 2, 12, 10, 12, 2, LinesCfg<Rad<12, 10, 12>, 2>::THREADS, LinesCfg<Rad<12, 10, 12>, 2>::SMEM_BYTES, launch_lines_1440_2},
    {1470, 0, 15, 7, 14, 4, LinesCfg<Rad<15, 7, 14>, 4>::THREADS, LinesCfg<Rad<15, 7, 14>, 4>::SMEM_BYTES, launch_lines_1470_0},
    {1470, 1, 14, 7, 15, 4, LinesCfg<Rad<14, 7, 15>, 4>::THREADS, LinesCfg<Rad<14, 7, 15>, 4>::SMEM_BYTES, launch_lines_1470_1},
    {1470, 2, 15, 7, 14, 2, LinesCfg<Rad<15, 7, 14>, 2>::THREADS, LinesCfg<Rad<15, 7, 14>, 2>::SMEM_BYTES, launch_lines_1470_2},
    {1500, 0, 15, 10, 10, 4, LinesCfg<Rad<15, 10, 10>, 4>::THREADS, LinesCfg<Rad<15, 10, 10>, 4>::SMEM_BYTES, launch_lines_1500_0},
    {1500, 1, 10, 10, 15, 4, LinesCfg<Rad<10, 10, 15>, 4>::THREADS, LinesCfg<Rad<10, 10, 15>, 4>::SMEM_BYTES, launch_lines_1500_1},
    {1500, 2, 15, 10, 10, 2, LinesCfg<Rad<15, 10, 10>, 2>::THREADS, LinesCfg<Rad<15, 10, 10>, 2>::SMEM_BYTES, launch_lines_1500_2},
    {1512, 0, 14, 9, 12, 4, LinesCfg<Rad<14, 9, 12>, 4>::THREADS, LinesCfg<Rad<14, 9, 12>, 4>::SMEM_BYTES, launch_lines_1512_0},
    {1512, 1, 12, 9, 14, 4, LinesCfg<Rad<12, 9, 14>, 4>::THREADS, LinesCfg<Rad<12, 9, 14>, 4>::SMEM_BYTES, launch_lines_1512_1},
    {1512, 2, 14, 9, 12, 2, LinesCfg<Rad<14, 9, 12>, 2>::THREADS, LinesCfg<Rad<14, 9, 12>, 2>::SMEM_BYTES, launch_lines_1512_2},
    {1536, 0, 16, 8, 12, 4, LinesCfg<Rad<16, 8, 12>, 4>::THREADS, LinesCfg<Rad<16, 8, 12>, 4>::SMEM_BYTES, launch_lines_1536_0},
    {1536, 1, 12, 8, 16, 4, LinesCfg<Rad<12, 8, 16>, 4>::THREADS, LinesCfg<Rad<12, 8, 16>, 4>::SMEM_BYTES, launch_lines_1536_1},
    {1536, 2, 16, 8, 12, 2, LinesCfg<Rad<16, 8, 12>, 2>::THREADS, LinesCfg<Rad<16, 8, 12>, 2>::SMEM_BYTES, launch_lines_1536_2},
    {1568, 0, 14, 8, 14, 4, LinesCfg<Rad<14, 8, 14>, 4>::THREADS, LinesCfg<Rad<14, 8, 14>, 4>::SMEM_BYTES, launch_lines_1568_0},
    {1568, 1, 8, 14, 14, 4, LinesCfg<Rad<8, 14, 14>, 4>::THREADS, LinesCfg<Rad<8, 14, 14>, 4>::SMEM_BYTES, launch_lines_1568_1},
    {1568, 2, 14, 8, 14, 2, LinesCfg<Rad<14, 8, 14>, 2>::THREADS, LinesCfg<Rad<14, 8, 14>, 2>::SMEM_BYTES, launch_lines_1568_2},
    {1575, 0, 15, 7, 15, 4, LinesCfg<Rad<15, 7, 15>, 4>::THREADS, LinesCfg<Rad<15, 7, 15>, 4>::SMEM_BYTES, launch_lines_1575_0},
    {1575, 1, 7, 15, 15, 4, LinesCfg<Rad<7, 15, 15>, 4>::THREADS, LinesCfg<Rad<7, 15, 15>, 4>::SMEM_BYTES, launch_lines_1575_1},
    {1575, 2, 15, 7, 15, 2, LinesCfg<Rad<15, 7, 15>, 2>::THREADS, LinesCfg<Rad<15, 7, 15>, 2>::SMEM_BYTES, launch_lines_1575_2},
    {1600, 0, 16, 10, 10, 4, LinesCfg<Rad<16, 10, 10>, 4>::THREADS, LinesCfg<Rad<16, 10, 10>, 4>::SMEM_BYTES, launch_lines_1600_0},
    {1600, 1, 10, 10, 16, 4, LinesCfg<Rad<10, 10, 16>, 4>::THREADS, LinesCfg<Rad<10, 10, 16>, 4>::SMEM_BYTES, launch_lines_1600_1},
    {1600, 2, 16, 10, 10, 2, LinesCfg<Rad<16, 10, 10>, 2>::THREADS, LinesCfg<Rad<16, 10, 10>, 2>::SMEM_BYTES, launch_lines_1600_2},
    {1620, 0, 15, 9, 12, 4, LinesCfg<Rad<15, 9, 12>, 4>::THREADS, LinesCfg<Rad<15, 9, 12>, 4>::SMEM_BYTES, launch_lines_1620_0},
    {1620, 1, 12, 9, 15, 4, LinesCfg<Rad<12, 9, 15>, 4>::THREADS, LinesCfg<Rad<12, 9, 15>, 4>::SMEM_BYTES, launch_lines_1620_1},
    {1620, 2, 15, 9, 12, 2, LinesCfg<Rad<15, 9, 12>, 2>::THREADS, LinesCfg<Rad<15, 9, 12>, 2>::SMEM_BYTES, launch_lines_1620_2},
    {1680, 0, 14, 10, 12, 4, LinesCfg<Rad<14, 10, 12>, 4>::THREADS, LinesCfg<Rad<14, 10, 12>, 4>::SMEM_BYTES, launch_lines_1680_0},
    {1680, 1, 12, 10, 14, 4, LinesCfg<Rad<12, 10, 14>, 4>::THREADS, LinesCfg<Rad<12, 10, 14>, 4>::SMEM_BYTES, launch_lines_1680_1},
    {1680, 2, 14, 10, 12, 2, LinesCfg<Rad<14, 10, 12>, 2>::THREADS, LinesCfg<Rad<14, 10, 12>, 2>::SMEM_BYTES, launch_lines_1680_2},
    {1728, 0, 12, 12, 12, 4, LinesCfg<Rad<12, 12, 12>, 4>::THREADS, LinesCfg<Rad<12, 12, 12>, 4>::SMEM_BYTES, launch_lines_1728_0},
    {1728, 1, 16, 9, 12, 4, LinesCfg<Rad<16, 9, 12>, 4>::THREADS, LinesCfg<Rad<16, 9, 12>, 4>::SMEM_BYTES, launch_lines_1728_1},
    {1728, 2, 12, 12, 12, 2, LinesCfg<Rad<12, 12, 12>, 2>::THREADS, LinesCfg<Rad<12, 12, 12>, 2>::SMEM_BYTES, launch_lines_1728_2},
    {1764, 0, 14, 9, 14, 4, LinesCfg<Rad<14, 9, 14>, 4>::THREADS, LinesCfg<Rad<14, 9, 14>, 4>::SMEM_BYTES, launch_lines_1764_0},
    {1764, 1, 9, 14, 14, 4, LinesCfg<Rad<9, 14, 14>, 4>::THREADS, LinesCfg<Rad<9, 14, 14>, 4>::SMEM_BYTES, launch_lines_1764_1},
    {1764, 2, 14, 9, 14, 2, LinesCfg<Rad<14, 9, 14>, 2>::THREADS, LinesCfg<Rad<14, 9, 14>, 2>::SMEM_BYTES, launch_lines_1764_2},
    {1792, 0, 16, 8, 14, 4, LinesCfg<Rad<16, 8, 14>, 4>::THREADS, LinesCfg<Rad<16, 8, 14>, 4>::SMEM_BYTES, launch_lines_1792_0},
    {1792, 1, 14, 8, 16, 4, LinesCfg<Rad<14, 8, 16>, 4>::THREADS, LinesCfg<Rad<14, 8, 16>, 4>::SMEM_BYTES, launch_lines_1792_1},
    {1792, 2, 16, 8, 14, 2, LinesCfg<Rad<16, 8, 14>, 2>::THREADS, LinesCfg<Rad<16, 8, 14>, 2>::SMEM_BYTES, launch_lines_1792_2},
    {1800, 0, 15, 10, 12, 4, LinesCfg<Rad<15, 10, 12>, 4>::THREADS, LinesCfg<Rad<15, 10, 12>, 4>::SMEM_BYTES, launch_lines_1800_0},
    {1800, 1, 12, 10, 15, 4, LinesCfg<Rad<12, 10, 15>, 4>::THREADS, LinesCfg<Rad<12, 10, 15>, 4>::SMEM_BYTES, launch_lines_1800_1},
    {1800, 2, 15, 10, 12, 2, LinesCfg<Rad<15, 10, 12>, 2>::THREADS, LinesCfg<Rad<15, 10, 12>, 2>::SMEM_BYTES, launch_lines_1800_2},
    {1890, 0, 15, 9, 14, 4, LinesCfg<Rad<15, 9, 14>, 4>::THREADS, LinesCfg<Rad<15, 9, 14>, 4>::SMEM_BYTES, launch_lines_1890_0},
    {1890, 1, 14, 9, 15, 4, LinesCfg<Rad<14, 9, 15>, 4>::THREADS, LinesCfg<Rad<14, 9, 15>, 4>::SMEM_BYTES, launch_lines_1890_1},
    {1890, 2, 15, 9, 14, 2, LinesCfg<Rad<15, 9, 14>, 2>::THREADS, LinesCfg<Rad<15, 9, 14>, 2>::SMEM_BYTES, launch_lines_1890_2},
    {1920, 0, 16, 10, 12, 4, LinesCfg<Rad<16, 10, 12>, 4>::THREADS, LinesCfg<Rad<16, 10, 12>, 4>::SMEM_BYTES, launch_lines_1920_0},
    {1920, 1, 12, 10, 16, 4, LinesCfg<Rad<12, 10, 16>, 4>::THREADS, LinesCfg<Rad<12, 10, 16>, 4>::SMEM_BYTES, launch_lines_1920_1},
    {1920, 2, 16, 10, 12, 2, LinesCfg<Rad<16, 10, 12>, 2>::THREADS, LinesCfg<Rad<16, 10, 12>, 2>::SMEM_BYTES, launch_lines_1920_2},
    {1960, 0, 14, 10, 14, 4, LinesCfg<Rad<14, 10, 14>, 4>::THREADS, LinesCfg<Rad<14, 10, 14>, 4>::SMEM_BYTES, launch_lines_1960_0},
    {1960, 1, 10, 14, 14, 4, LinesCfg<Rad<10, 14, 14>, 4>::THREADS, LinesCfg<Rad<10, 14, 14>, 4>::SMEM_BYTES, launch_lines_1960_1},
    {1960, 2, 14, 10, 14, 2, LinesCfg<Rad<14, 10, 14>, 2>::THREADS, LinesCfg<Rad<14, 10, 14>, 2>::SMEM_BYTES, launch_lines_1960_2},
    {2016, 0, 14, 12, 12, 4, LinesCfg<Rad<14, 12, 12>, 4>::THREADS, LinesCfg<Rad<14, 12, 12>, 4>::SMEM_BYTES, launch_lines_2016_0},
    {2016, 1, 12, 12, 14, 4, LinesCfg<Rad<12, 12, 14>, 4>::THREADS, LinesCfg<Rad<12, 12, 14>, 4>::SMEM_BYTES, launch_lines_2016_1},
    {2016, 2, 14, 12, 12, 2, LinesCfg<Rad<14, 12, 12>, 2>::THREADS, LinesCfg<Rad<14, 12, 12>, 2>::SMEM_BYTES, launch_lines_2016_2},
    {2025, 0, 15, 9, 15, 4, LinesCfg<Rad<15, 9, 15>, 4>::THREADS, LinesCfg<Rad<15, 9, 15>, 4>::SMEM_BYTES, launch_lines_2025_0},
    {2025, 1, 9, 15, 15, 4, LinesCfg<Rad<9, 15, 15>, 4>::THREADS, LinesCfg<Rad<9, 15, 15>, 4>::SMEM_BYTES, launch_lines_2025_1},
    {2025, 2, 15, 9, 15, 2, LinesCfg<Rad<15, 9, 15>, 2>::THREADS, LinesCfg<Rad<15, 9, 15>, 2>::SMEM_BYTES, launch_lines_2025_2},
    {2048, 0, 16, 8, 16, 4, LinesCfg<Rad<16, 8, 16>, 4>::THREADS, LinesCfg<Rad<16, 8, 16>, 4>::SMEM_BYTES, launch_lines_2048_0},
    {2048, 1, 8, 16, 16, 4, LinesCfg<Rad<8, 16, 16>, 4>::THREADS, LinesCfg<Rad<8, 16, 16>, 4>::SMEM_BYTES, launch_lines_2048_1},
    {2048, 2, 16, 8, 16, 2, LinesCfg<Rad<16, 8, 16>, 2>::THREADS, LinesCfg<Rad<16, 8, 16>, 2>::SMEM_BYTES, launch_lines_2048_2},
    {2100, 0, 15, 10, 14, 4, LinesCfg<Rad<15, 10, 14>, 4>::THREADS, LinesCfg<Rad<15, 10, 14>, 4>::SMEM_BYTES, launch_lines_2100_0},
    {2100, 1, 14, 10, 15, 4, LinesCfg<Rad<14, 10, 15>, 4>::THREADS, LinesCfg<Rad<14, 10, 15>, 4>::SMEM_BYTES, launch_lines_2100_1},
    {2100, 2, 15, 10, 14, 2, LinesCfg<Rad<15, 10, 14>, 2>::THREADS, LinesCfg<Rad<15, 10, 14>, 2>::SMEM_BYTES, launch_lines_2100_2},
    {2160, 0, 15, 12, 12, 4, LinesCfg<Rad<15, 12, 12>, 4>::THREADS, LinesCfg<Rad<15, 12, 12>, 4>::SMEM_BYTES, launch_lines_2160_0},
    {2160, 1, 12, 12, 15, 4, LinesCfg<Rad<12, 12, 15>, 4>::THREADS, LinesCfg<Rad<12, 12, 15>, 4>::SMEM_BYTES, launch_lines_2160_1},
    {2160, 2, 15, 12, 12, 2, LinesCfg<Rad<15, 12, 12>, 2>::THREADS, LinesCfg<Rad<15, 12, 12>, 2>::SMEM_BYTES, launch_lines_2160_2},
    {2240, 0, 16, 10, 14, 4, LinesCfg<Rad<16, 10, 14>, 4>::THREADS, LinesCfg<Rad<16, 10, 14>, 4>::SMEM_BYTES, launch_lines_2240_0},
    {2240, 1, 14, 10, 16, 4, LinesCfg<Rad<14, 10, 16>, 4>::THREADS, LinesCfg<Rad<14, 10, 16>, 4>::SMEM_BYTES, launch_lines_2240_1},
    {2240, 2, 16, 10, 14, 2, LinesCfg<Rad<16, 10, 14>, 2>::THREADS, LinesCfg<Rad<16, 10, 14>, 2>::SMEM_BYTES, launch_lines_2240_2},
    {2250, 0, 15, 10, 15, 4, LinesCfg<Rad<15, 10, 15>, 4>::THREADS, LinesCfg<Rad<15, 10, 15>, 4>::SMEM_BYTES, launch_lines_2250_0},
    {2250, 1, 10, 15, 15, 4, LinesCfg<Rad<10, 15, 15>, 4>::THREADS, LinesCfg<Rad<10, 15, 15>, 4>::SMEM_BYTES, launch_lines_2250_1},
    {2250, 2, 15, 10, 15, 2, LinesCfg<Rad<15, 10, 15>, 2>::THREADS, LinesCfg<Rad<15, 10, 15>, 2>::SMEM_BYTES, launch_lines_2250_2},
    {2304, 0, 16, 12, 12, 4, LinesCfg<Rad<16, 12, 12>, 4>::THREADS, LinesCfg<Rad<16, 12, 12>, 4>::SMEM_BYTES, launch_lines_2304_0},
    {2304, 1, 12, 12, 16, 4, LinesCfg<Rad<12, 12, 16>, 4>::THREADS, LinesCfg<Rad<12, 12, 16>, 4>::SMEM_BYTES, launch_lines_2304_1},
    {2304, 2, 16, 12, 12, 2, LinesCfg<Rad<16, 12, 12>, 2>::THREADS, LinesCfg<Rad<16, 12, 12>, 2>::SMEM_BYTES, launch_lines_2304_2},
    {2352, 0, 14, 12, 14, 4, LinesCfg<Rad<14, 12, 14>, 4>::THREADS, LinesCfg<Rad<14, 12, 14>, 4>::SMEM_BYTES, launch_lines_2352_0},
    {2352, 1, 12, 14, 14, 4, LinesCfg<Rad<12, 14, 14>, 4>::THREADS, LinesCfg<Rad<12, 14, 14>, 4>::SMEM_BYTES, launch_lines_2352_1},
    {2352, 2, 14, 12, 14, 2, LinesCfg<Rad<14, 12, 14>, 2>::THREADS, LinesCfg<Rad<14, 12, 14>, 2>::SMEM_BYTES, launch_lines_2352_2},
    {2400, 0, 16, 10, 15, 4, LinesCfg<Rad<16, 10, 15>, 4>::THREADS, LinesCfg<Rad<16, 10, 15>, 4>::SMEM_BYTES, launch_lines_2400_0},
    {2400, 1, 15, 10, 16, 4, LinesCfg<Rad<15, 10, 16>, 4>::THREADS, LinesCfg<Rad<15, 10, 16>, 4>::SMEM_BYTES, launch_lines_2400_1},
    {2400, 2, 16, 10, 15, 2, LinesCfg<Rad<16, 10, 15>, 2>::THREADS, LinesCfg<Rad<16, 10, 15>, 2>::SMEM_BYTES, launch_lines_2400_2},
    {2520, 0, 15, 12, 14, 4, LinesCfg<Rad<15, 12, 14>, 4>::THREADS, LinesCfg<Rad<15, 12, 14>, 4>::SMEM_BYTES, launch_lines_2520_0},
    {2520, 1, 14, 12, 15, 4, LinesCfg<Rad<14, 12, 15>, 4>::THREADS, LinesCfg<Rad<14, 12, 15>, 4>::SMEM_BYTES, launch_lines_2520_1},
    {2520, 2, 15, 12, 14, 2, LinesCfg<Rad<15, 12, 14>, 2>::THREADS, LinesCfg<Rad<15, 12, 14>, 2>::SMEM_BYTES, launch_lines_2520_2},
    {2560, 0, 16, 10, 16, 4, LinesCfg<Rad<16, 10, 16>, 4>::THREADS, LinesCfg<Rad<16, 10, 16>, 4>::SMEM_BYTES, launch_lines_2560_0},
    {2560, 1, 10, 16, 16, 4, LinesCfg<Rad<10, 16, 16>, 4>::THREADS, LinesCfg<Rad<10, 16, 16>, 4>::SMEM_BYTES, launch_lines_2560_1},
    {2560, 2, 16, 10, 16, 2, LinesCfg<Rad<16, 10, 16>, 2>::THREADS, LinesCfg<Rad<16, 10, 16>, 2>::SMEM_BYTES, launch_lines_2560_2},
    {2688, 0, 16, 12, 14, 4, LinesCfg<Rad<16, 12, 14>, 4>::THREADS, LinesCfg<Rad<16, 12, 14>, 4>::SMEM_BYTES, launch_lines_2688_0},
    {2688, 1, 14, 12, 16, 4, LinesCfg<Rad<14, 12, 16>, 4>::THREADS, LinesCfg<Rad<14, 12, 16>, 4>::SMEM_BYTES, launch_lines_2688_1},
    {2688, 2, 16, 12, 14, 2, LinesCfg<Rad<16, 12, 14>, 2>::THREADS, LinesCfg<Rad<16, 12, 14>, 2>::SMEM_BYTES, launch_lines_2688_2},
    {2700, 0, 15, 12, 15, 4, LinesCfg<Rad<15, 12, 15>, 4>::THREADS, LinesCfg<Rad<15, 12, 15>, 4>::SMEM_BYTES, launch_lines_2700_0},
    {2700, 1, 12, 15, 15, 4, LinesCfg<Rad<12, 15, 15>, 4>::THREADS, LinesCfg<Rad<12, 15, 15>, 4>::SMEM_BYTES, launch_lines_2700_1},
    {2700, 2, 15, 12, 15, 2, LinesCfg<Rad<15, 12, 15>, 2>::THREADS, LinesCfg<Rad<15, 12, 15>, 2>::SMEM_BYTES, launch_lines_2700_2},
    {2744, 0, 14, 14, 14, 4, LinesCfg<Rad<14, 14, 14>, 4>::THREADS, LinesCfg<Rad<14, 14, 14>, 4>::SMEM_BYTES, launch_lines_2744_0},
    {2744, 1, 14, 14, 14, 2, LinesCfg<Rad<14, 14, 14>, 2>::THREADS, LinesCfg<Rad<14, 14, 14>, 2>::SMEM_BYTES, launch_lines_2744_1},
    {2880, 0, 16, 12, 15, 4, LinesCfg<Rad<16, 12, 15>, 4>::THREADS, LinesCfg<Rad<16, 12, 15>, 4>::SMEM_BYTES, launch_lines_2880_0},
    {2880, 1, 15, 12, 16, 4, LinesCfg<Rad<15, 12, 16>, 4>::THREADS, LinesCfg<Rad<15, 12, 16>, 4>::SMEM_BYTES, launch_lines_2880_1},
    {2880, 2, 16, 12, 15, 2, LinesCfg<Rad<16, 12, 15>, 2>::THREADS, LinesCfg<Rad<16, 12, 15>, 2>::SMEM_BYTES, launch_lines_2880_2},
    {2940, 0, 15, 14, 14, 4, LinesCfg<Rad<15, 14, 14>, 4>::THREADS, LinesCfg<Rad<15, 14, 14>, 4>::SMEM_BYTES, launch_lines_2940_0},
    {2940, 1, 14, 14, 15, 4, LinesCfg<Rad<14, 14, 15>, 4>::THREADS, LinesCfg<Rad<14, 14, 15>, 4>::SMEM_BYTES, launch_lines_2940_1},
    {2940, 2, 15, 14, 14, 2, LinesCfg<Rad<15, 14, 14>, 2>::THREADS, LinesCfg<Rad<15, 14, 14>, 2>::SMEM_BYTES, launch_lines_2940_2},
    {3072, 0, 16, 12, 16, 2, LinesCfg<Rad<16, 12, 16>, 2>::THREADS, LinesCfg<Rad<16, 12, 16>, 2>::SMEM_BYTES, launch_lines_3072_0},
    {3072, 1, 12, 16, 16, 2, LinesCfg<Rad<12, 16, 16>, 2>::THREADS, LinesCfg<Rad<12, 16, 16>, 2>::SMEM_BYTES, launch_lines_3072_1},
    {3136, 0, 16, 14, 14, 2, LinesCfg<Rad<16, 14, 14>, 2>::THREADS, LinesCfg<Rad<16, 14, 14>, 2>::SMEM_BYTES, launch_lines_3136_0},
    {3136, 1, 14, 14, 16, 2, LinesCfg<Rad<14, 14, 16>, 2>::THREADS, LinesCfg<Rad<14, 14, 16>, 2>::SMEM_BYTES, launch_lines_3136_1},
    {3150, 0, 15, 14, 15, 2, LinesCfg<Rad<15, 14, 15>, 2>::THREADS, LinesCfg<Rad<15, 14, 15>, 2>::SMEM_BYTES, launch_lines_3150_0},
    {3150, 1, 14, 15, 15, 2, LinesCfg<Rad<14, 15, 15>, 2>::THREADS, LinesCfg<Rad<14, 15, 15>, 2>::SMEM_BYTES, launch_lines_3150_1},
    {3360, 0, 16, 14, 15, 2, LinesCfg<Rad<16, 14, 15>, 2>::THREADS, LinesCfg<Rad<16, 14, 15>, 2>::SMEM_BYTES, launch_lines_3360_0},
    {3360, 1, 15, 14, 16, 2, LinesCfg<Rad<15, 14, 16>, 2>::THREADS, LinesCfg<Rad<15, 14, 16>, 2>::SMEM_BYTES, launch_lines_3360_1},
    {3375, 0, 15, 15, 15, 2, LinesCfg<Rad<15, 15, 15>, 2>::THREADS, LinesCfg<Rad<15, 15, 15>, 2>::SMEM_BYTES, launch_lines_3375_0},
    {3584, 0, 16, 14, 16, 2, LinesCfg<Rad<16, 14, 16>, 2>::THREADS, LinesCfg<Rad<16, 14, 16>, 2>::SMEM_BYTES, launch_lines_3584_0},
    {3584, 1, 14, 16, 16, 2, LinesCfg<Rad<14, 16, 16>, 2>::THREADS, LinesCfg<Rad<14, 16, 16>, 2>::SMEM_BYTES, launch_lines_3584_1},
    {3600, 0, 16, 15, 15, 2, LinesCfg<Rad<16, 15, 15>, 2>::THREADS, LinesCfg<Rad<16, 15, 15>, 2>::SMEM_BYTES, launch_lines_3600_0},
    {3600, 1, 15, 15, 16, 2, LinesCfg<Rad<15, 15, 16>, 2>::THREADS, LinesCfg<Rad<15, 15, 16>, 2>::SMEM_BYTES, launch_lines_3600_1},
    {3840, 0, 16, 15, 16, 2, LinesCfg<Rad<16, 15, 16>, 2>::THREADS, LinesCfg<Rad<16, 15, 16>, 2>::SMEM_BYTES, launch_lines_3840_0},
    {3840, 1, 15, 16, 16, 2, LinesCfg<Rad<15, 16, 16>, 2>::THREADS, LinesCfg<Rad<15, 16, 16>, 2>::SMEM_BYTES, launch_lines_3840_1},
    {4096, 0, 16, 16, 16, 2, LinesCfg<Rad<16, 16, 16>, 2>::THREADS, LinesCfg<Rad<16, 16, 16>, 2>::SMEM_BYTES, launch_lines_4096_0},
};
static const XPlan kXPlans[] = {
    {2, 0, 2, 1, 1, 32, XCfg<Rad<2, 1, 1>, 32>::THREADS, XCfg<Rad<2, 1, 1>, 32>::SMEM_BYTES, launch_x_2_0},
    {3, 0, 3, 1, 1, 32, XCfg<Rad<3, 1, 1>, 32>::THREADS, XCfg<Rad<3, 1, 1>, 32>::SMEM_BYTES, launch_x_3_0},
    {4, 0, 2, 2, 1, 32, XCfg<Rad<2, 2, 1>, 32>::THREADS, XCfg<Rad<2, 2, 1>, 32>::SMEM_BYTES, launch_x_4_0},
    {5, 0, 5, 1, 1, 16, XCfg<Rad<5, 1, 1>, 16>::THREADS, XCfg<Rad<5, 1, 1>, 16>::SMEM_BYTES, launch_x_5_0},
    {6, 0, 3, 2, 1, 32, XCfg<Rad<3, 2, 1>, 32>::THREADS, XCfg<Rad<3, 2, 1>, 32>::SMEM_BYTES, launch_x_6_0},
    {7, 0, 7, 1, 1, 16, XCfg<Rad<7, 1, 1>, 16>::THREADS, XCfg<Rad<7, 1, 1>, 16>::SMEM_BYTES, launch_x_7_0},
    {8, 0, 4, 2, 1, 16, XCfg<Rad<4, 2, 1>, 16>::THREADS, XCfg<Rad<4, 2, 1>, 16>::SMEM_BYTES, launch_x_8_0},
    {9, 0, 3, 3, 1, 32, XCfg<Rad<3, 3, 1>, 32>::THREADS, XCfg<Rad<3, 3, 1>, 32>::SMEM_BYTES, launch_x_9_0},
    {10, 0, 5, 2, 1, 16, XCfg<Rad<5, 2, 1>, 16>::THREADS, XCfg<Rad<5, 2, 1>, 16>::SMEM_BYTES, launch_x_10_0},
    {12, 0, 4, 3, 1, 16, XCfg<Rad<4, 3, 1>, 16>::THREADS, XCfg<Rad<4, 3, 1>, 16>::SMEM_BYTES, launch_x_12_0},
    {14, 0, 7, 2, 1, 16, XCfg<Rad<7, 2, 1>, 16>::THREADS, XCfg<Rad<7, 2, 1>, 16>::SMEM_BYTES, launch_x_14_0},
    {15, 0, 5, 3, 1, 16, XCfg<Rad<5, 3, 1>, 16>::THREADS, XCfg<Rad<5, 3, 1>, 16>::SMEM_BYTES, launch_x_15_0},
    {16, 0, 4, 4, 1, 16, XCfg<Rad<4, 4, 1>, 16>::THREADS, XCfg<Rad<4, 4, 1>, 16>::SMEM_BYTES, launch_x_16_0},
    {18, 0, 6, 3, 1, 16, XCfg<Rad<6, 3, 1>, 16>::THREADS, XCfg<Rad<6, 3, 1>, 16>::SMEM_BYTES, launch_x_18_0},
    {20, 0, 5, 4, 1, 16, XCfg<Rad<5, 4, 1>, 16>::THREADS, XCfg<Rad<5, 4, 1>, 16>::SMEM_BYTES, launch_x_20_0},
    {21, 0, 7, 3, 1, 16, XCfg<Rad<7, 3, 1>, 16>::THREADS, XCfg<Rad<7, 3, 1>, 16>::SMEM_BYTES, launch_x_21_0},
    {24, 0, 6, 4, 1, 16, XCfg<Rad<6, 4, 1>, 16>::THREADS, XCfg<Rad<6, 4, 1>, 16>::SMEM_BYTES, launch_x_24_0},
    {25, 0, 5, 5, 1, 16, XCfg<Rad<5, 5, 1>, 16>::THREADS, XCfg<Rad<5, 5, 1>, 16>::SMEM_BYTES, launch_x_25_0},
    {27, 0, 9, 3, 1, 8, XCfg<Rad<9, 3, 1>, 8>::THREADS, XCfg<Rad<9, 3, 1>, 8>::SMEM_BYTES, launch_x_27_0},
    {28, 0, 7, 4, 1, 16, XCfg<Rad<7, 4, 1>, 16>::THREADS, XCfg<Rad<7, 4, 1>, 16>::SMEM_BYTES, launch_x_28_0},
    {30, 0, 6, 5, 1, 16, XCfg<Rad<6, 5, 1>, 16>::THREADS, XCfg<Rad<6, 5, 1>, 16>::SMEM_BYTES, launch_x_30_0},
    {32, 0, 8, 4, 1, 8, XCfg<Rad<8, 4, 1>, 8>::THREADS, XCfg<Rad<8, 4, 1>, 8>::SMEM_BYTES, launch_x_32_0},
    {35, 0, 7, 5, 1, 16, XCfg<Rad<7, 5, 1>, 16>::THREADS, XCfg<Rad<7, 5, 1>, 16>::SMEM_BYTES, launch_x_35_0},
    {36, 0, 6, 6, 1, 16, XCfg<Rad<6, 6, 1>, 16>::THREADS, XCfg<Rad<6, 6, 1>, 16>::SMEM_BYTES, launch_x_36_0},
    {40, 0, 8, 5, 1, 8, XCfg<Rad<8, 5, 1>, 8>::THREADS, XCfg<Rad<8, 5, 1>, 8>::SMEM_BYTES, launch_x_40_0},
    {42, 0, 7, 6, 1, 16, XCfg<Rad<7, 6, 1>, 16>::THREADS, XCfg<Rad<7, 6, 1>, 16>::SMEM_BYTES, launch_x_42_0},
    {45, 0, 9, 5, 1, 8, XCfg<Rad<9, 5, 1>, 8>::THREADS, XCfg<Rad<9, 5, 1>, 8>::SMEM_BYTES, launch_x_45_0},
    {48, 0, 8, 6, 1, 8, XCfg<Rad<8, 6, 1>, 8>::THREADS, XCfg<Rad<8, 6, 1>, 8>::SMEM_BYTES, launch_x_48_0},
    {49, 0, 7, 7, 1, 16, XCfg<Rad<7, 7, 1>, 16>::THREADS, XCfg<Rad<7, 7, 1>, 16>::SMEM_BYTES, launch_x_49_0},
    {50, 0, 10, 5, 1, 8, XCfg<Rad<10, 5, 1>, 8>::THREADS, XCfg<Rad<10, 5, 1>, 8>::SMEM_BYTES, launch_x_50_0},
    {54, 0, 9, 6, 1, 8, XCfg<Rad<9, 6, 1>, 8>::THREADS, XCfg<Rad<9, 6, 1>, 8>::SMEM_BYTES, launch_x_54_0},
    {56, 0, 8, 7, 1, 8, XCfg<Rad<8, 7, 1>, 8>::THREADS, XCfg<Rad<8, 7, 1>, 8>::SMEM_BYTES, launch_x_56_0},
    {60, 0, 10, 6, 1, 8, XCfg<Rad<10, 6, 1>, 8>::THREADS, XCfg<Rad<10, 6, 1>, 8>::SMEM_BYTES, launch_x_60_0},
    {63, 0, 9, 7, 1, 8, XCfg<Rad<9, 7, 1>, 8>::THREADS, XCfg<Rad<9, 7, 1>, 8>::SMEM_BYTES, launch_x_63_0},
    {64, 0, 8, 8, 1, 8, XCfg<Rad<8, 8, 1>, 8>::THREADS, XCfg<Rad<8, 8, 1>, 8>::SMEM_BYTES, launch_x_64_0},
    {70, 0, 10, 7, 1, 8, XCfg<Rad<10, 7, 1>, 8>::THREADS, XCfg<Rad<10, 7, 1>, 8>::SMEM_BYTES, launch_x_70_0},
    {72, 0, 9, 8, 1, 8, XCfg<Rad<9, 8, 1>, 8>::THREADS, XCfg<Rad<9, 8, 1>, 8>::SMEM_BYTES, launch_x_72_0},
    {75, 0, 15, 5, 1, 8, XCfg<Rad<15, 5, 1>, 8>::THREADS, XCfg<Rad<15, 5, 1>, 8>::SMEM_BYTES, launch_x_75_0},
    {80, 0, 10, 8, 1, 8, XCfg<Rad<10, 8, 1>, 8>::THREADS, XCfg<Rad<10, 8, 1>, 8>::SMEM_BYTES, launch_x_80_0},
    {81, 0, 9, 9, 1, 8, XCfg<Rad<9, 9, 1>, 8>::THREADS, XCfg<Rad<9, 9, 1>, 8>::SMEM_BYTES, launch_x_81_0},
    {84, 0, 12, 7, 1, 8, XCfg<Rad<12, 7, 1>, 8>::THREADS, XCfg<Rad<12, 7, 1>, 8>::SMEM_BYTES, launch_x_84_0},
    {90, 0, 10, 9, 1, 8, XCfg<Rad<10, 9, 1>, 8>::THREADS, XCfg<Rad<10, 9, 1>, 8>::SMEM_BYTES, launch_x_90_0},
    {96, 0, 12, 8, 1, 8, XCfg<Rad<12, 8, 1>, 8>::THREADS, XCfg<Rad<12, 8, 1>, 8>::SMEM_BYTES, launch_x_96_0},
    {96, 1, 8, 12, 1, 8, XCfg<Rad<8, 12, 1>, 8>::THREADS, XCfg<Rad<8, 12, 1>, 8>::SMEM_BYTES, launch_x_96_1},
    {98, 0, 14, 7, 1, 8, XCfg<Rad<14, 7, 1>, 8>::THREADS, XCfg<Rad<14, 7, 1>, 8>::SMEM_BYTES, launch_x_98_0},
    {98, 1, 7, 14, 1, 8, XCfg<Rad<7, 14, 1>, 8>::THREADS, XCfg<Rad<7, 14, 1>, 8>::SMEM_BYTES, launch_x_98_1},
    {100, 0, 10, 10, 1, 8, XCfg<Rad<10, 10, 1>, 8>::THREADS, XCfg<Rad<10, 10, 1>, 8>::SMEM_BYTES, launch_x_100_0},
    {105, 0, 15, 7, 1, 8, XCfg<Rad<15, 7, 1>, 8>::THREADS, XCfg<Rad<15, 7, 1>, 8>::SMEM_BYTES, launch_x_105_0},
    {105, 1, 7, 15, 1, 8, XCfg<Rad<7, 15, 1>, 8>::THREADS, XCfg<Rad<7, 15, 1>, 8>::SMEM_BYTES, launch_x_105_1},
    {108, 0, 12, 9, 1, 8, XCfg<Rad<12, 9, 1>, 8>::THREADS, XCfg<Rad<12, 9, 1>, 8>::SMEM_BYTES, launch_x_108_0},
    {108, 1, 9, 12, 1, 8, XCfg<Rad<9, 12, 1>, 8>::THREADS, XCfg<Rad<9, 12, 1>, 8>::SMEM_BYTES, launch_x_108_1},
    {112, 0, 14, 8, 1, 8, XCfg<Rad<14, 8, 1>, 8>::THREADS, XCfg<Rad<14, 8, 1>, 8>::SMEM_BYTES, launch_x_112_0},
    {112, 1, 8, 14, 1, 8, XCfg<Rad<8, 14, 1>, 8>::THREADS, XCfg<Rad<8, 14, 1>, 8>::SMEM_BYTES, launch_x_112_1},
    {120, 0, 12, 10, 1, 8, XCfg<Rad<12, 10, 1>, 8>::THREADS, XCfg<Rad<12, 10, 1>, 8>::SMEM_BYTES, launch_x_120_0},
    {120, 1, 10, 12, 1, 8, XCfg<Rad<10, 12, 1>, 8>::THREADS, XCfg<Rad<10, 12, 1>, 8>::SMEM_BYTES, launch_x_120_1},
    {125, 0, 5, 5, 5, 4, XCfg<Rad<5, 5, 5>, 4>::THREADS, XCfg<Rad<5, 5, 5>, 4>::SMEM_BYTES, launch_x_125_0},
    {126, 0, 14, 9, 1, 8, XCfg<Rad<14, 9, 1>, 8>::THREADS, XCfg<Rad<14, 9, 1>, 8>::SMEM_BYTES, launch_x_126_0},
    {126, 1, 9, 14, 1, 8, XCfg<Rad<9, 14, 1>, 8>::THREADS, XCfg<Rad<9, 14, 1>, 8>::SMEM_BYTES, launch_x_126_1},
    {128, 0, 16, 8, 1, 4, XCfg<Rad<16, 8, 1>, 4>::THREADS, XCfg<Rad<16, 8, 1>, 4>::SMEM_BYTES, launch_x_128_0},
    {128, 1, 8, 16, 1, 4, XCfg<Rad<8, 16, 1>, 4>::THREADS, XCfg<Rad<8, 16, 1>, 4>::SMEM_BYTES, launch_x_128_1},
    {135, 0, 15, 9, 1, 8, XCfg<Rad<15, 9, 1>, 8>::THREADS, XCfg<Rad<15, 9, 1>, 8>::SMEM_BYTES, launch_x_135_0},
    {135, 1, 9, 15, 1, 8, XCfg<Rad<9, 15, 1>, 8>::THREADS, XCfg<Rad<9, 15, 1>, 8>::SMEM_BYTES, launch_x_135_1},
    {140, 0, 14, 10, 1, 8, XCfg<Rad<14, 10, 1>, 8>::THREADS, XCfg<Rad<14, 10, 1>, 8>::SMEM_BYTES, launch_x_140_0},
    {140, 1, 10, 14, 1, 8, XCfg<Rad<10, 14, 1>, 8>::THREADS, XCfg<Rad<10, 14, 1>, 8>::SMEM_BYTES, launch_x_140_1},
    {144, 0, 12, 12, 1, 8, XCfg<Rad<12, 12, 1>, 8>::THREADS, XCfg<Rad<12, 12, 1>, 8>::SMEM_BYTES, launch_x_144_0},
    {147, 0, 7, 3, 7, 2, XCfg<Rad<7, 3, 7>, 2>::THREADS, XCfg<Rad<7, 3, 7>, 2>::SMEM_BYTES, launch_x_147_0},
    {147, 1, 3, 7, 7, 2, XCfg<Rad<3, 7, 7>, 2>::THREADS, XCfg<Rad<3, 7, 7>, 2>::SMEM_BYTES, launch_x_147_1},
    {150, 0, 15, 10, 1, 8, XCfg<Rad<15, 10, 1>, 8>::THREADS, XCfg<Rad<15, 10, 1>, 8>::SMEM_BYTES, launch_x_150_0},
    {150, 1, 10, 15, 1, 8, XCfg<Rad<10, 15, 1>, 8>::THREADS, XCfg<Rad<10, 15, 1>, 8>::SMEM_BYTES, launch_x_150_1},
    {160, 0, 16, 10, 1, 4, XCfg<Rad<16, 10, 1>, 4>::THREADS, XCfg<Rad<16, 10, 1>, 4>::SMEM_BYTES, launch_x_160_0},
    {160, 1, 10, 16, 1, 4, XCfg<Rad<10, 16, 1>, 4>::THREADS, XCfg<Rad<10, 16, 1>, 4>::SMEM_BYTES, launch_x_160_1},
    {162, 0, 9, 3, 6, 2, XCfg<Rad<9, 3, 6>, 2>::THREADS, XCfg<Rad<9, 3, 6>, 2>::SMEM_BYTES, launch_x_162_0},
    {162, 1, 6, 3, 9, 2, XCfg<Rad<6, 3, 9>, 2>::THREADS, XCfg<Rad<6, 3, 9>, 2>::SMEM_BYTES, launch_x_162_1},
    {168, 0, 14, 12, 1, 8, XCfg<Rad<14, 12, 1>, 8>::THREADS, XCfg<Rad<14, 12, 1>, 8>::SMEM_BYTES, launch_x_168_0},
    {168, 1, 12, 14, 1, 8, XCfg<Rad<12, 14, 1>, 8>::THREADS, XCfg<Rad<12, 14, 1>, 8>::SMEM_BYTES, launch_x_168_1},
    {175, 0, 7, 5, 5, 2, XCfg<Rad<7, 5, 5>, 2>::THREADS, XCfg<Rad<7, 5, 5>, 2>::SMEM_BYTES, launch_x_175_0},
    {175, 1, 5, 5, 7, 2, XCfg<Rad<5, 5, 7>, 2>::THREADS, XCfg<Rad<5, 5, 7>, 2>::SMEM_BYTES, launch_x_175_1},
    {180, 0, 15, 12, 1, 8, XCfg<Rad<15, 12, 1>, 8>::THREADS, XCfg<Rad<15, 12, 1>, 8>::SMEM_BYTES, launch_x_180_0},
    {180, 1, 12, 15, 1, 8, XCfg<Rad<12, 15, 1>, 8>::THREADS, XCfg<Rad<12, 15, 1>, 8>::SMEM_BYTES, launch_x_180_1},
    {189, 0, 9, 3, 7, 2, XCfg<Rad<9, 3, 7>, 2>::THREADS, XCfg<Rad<9, 3, 7>, 2>::SMEM_BYTES, launch_x_189_0},
    {189, 1, 7, 3, 9, 2, XCfg<Rad<7, 3, 9>, 2>::THREADS, XCfg<Rad<7, 3, 9>, 2>::SMEM_BYTES, launch_x_189_1},
    {192, 0, 16, 12, 1, 4, XCfg<Rad<16, 12, 1>, 4>::THREADS, XCfg<Rad<16, 12, 1>, 4>::SMEM_BYTES, launch_x_192_0},
    {192, 1, 12, 16, 1, 4, XCfg<Rad<12, 16, 1>, 4>::THREADS, XCfg<Rad<12, 16, 1>, 4>::SMEM_BYTES, launch_x_192_1},
    {196, 0, 14, 14, 1, 8, XCfg<Rad<14, 14, 1>, 8>::THREADS, XCfg<Rad<14, 14, 1>, 8>::SMEM_BYTES, launch_x_196_0},
    {200, 0, 8, 5, 5, 2, XCfg<Rad<8, 5, 5>, 2>::THREADS, XCfg<Rad<8, 5, 5>, 2>::SMEM_BYTES, launch_x_200_0},
    {200, 1, 5, 5, 8, 2, XCfg<Rad<5, 5, 8>, 2>::THREADS, XCfg<Rad<5, 5, 8>, 2>::SMEM_BYTES, launch_x_200_1},
    {210, 0, 15, 14, 1, 8, XCfg<Rad<15, 14, 1>, 8>::THREADS, XCfg<Rad<15, 14, 1>, 8>::SMEM_BYTES, launch_x_210_0},
    {210, 1, 14, 15, 1, 8, XCfg<Rad<14, 15, 1>, 8>::THREADS, XCfg<Rad<14, 15, 1>, 8>::SMEM_BYTES, launch_x_210_1},
    {216, 0, 6, 6, 6, 2, XCfg<Rad<6, 6, 6>, 2>::THREADS, XCfg<Rad<6, 6, 6>, 2>::SMEM_BYTES, launch_x_216_0},
    {216, 1, 9, 4, 6, 2, XCfg<Rad<9, 4, 6>, 2>::THREADS, XCfg<Rad<9, 4, 6>, 2>::SMEM_BYTES, launch_x_216_1},
    {224, 0, 16, 14, 1, 4, XCfg<Rad<16, 14, 1>, 4>::THREADS, XCfg<Rad<16, 14, 1>, 4>::SMEM_BYTES, launch_x_224_0},
    {224, 1, 14, 16, 1, 4, XCfg<Rad<14, 16, 1>, 4>::THREADS, XCfg<Rad<14, 16, 1>, 4>::SMEM_BYTES, launch_x_224_1},
    {225, 0, 15, 15, 1, 8, XCfg<Rad<15, 15, 1>, 8>::THREADS, XCfg<Rad<15, 15, 1>, 8>::SMEM_BYTES, launch_x_225_0},
    {240, 0, 16, 15, 1, 4, XCfg<Rad<16, 15, 1>, 4>::THREADS, XCfg<Rad<16, 15, 1>, 4>::SMEM_BYTES, launch_x_240_0},
    {240, 1, 15, 16, 1, 4, XCfg<Rad<15, 16, 1>, 4>::THREADS, XCfg<Rad<15, 16, 1>, 4>::SMEM_BYTES, launch_x_240_1},
    {243, 0, 9, 3, 9, 2, XCfg<Rad<9, 3, 9>, 2>::THREADS, XCfg<Rad<9, 3, 9>, 2>::SMEM_BYTES, launch_x_243_0},
    {243, 1, 3, 9, 9, 2, XCfg<Rad<3, 9, 9>, 2>::THREADS, XCfg<Rad<3, 9, 9>, 2>::SMEM_BYTES, launch_x_243_1},
    {245, 0, 7, 5, 7, 2, XCfg<Rad<7, 5, 7>, 2>::THREADS, XCfg<Rad<7, 5, 7>, 2>::SMEM_BYTES, launch_x_245_0},
    {245, 1, 5, 7, 7, 2, XCfg<Rad<5, 7, 7>, 2>::THREADS, XCfg<Rad<5, 7, 7>, 2>::SMEM_BYTES, launch_x_245_1},
    {250, 0, 10, 5, 5, 2, XCfg<Rad<10, 5, 5>, 2>::THREADS, XCfg<Rad<10, 5, 5>, 2>::SMEM_BYTES, launch_x_250_0},
    {250, 1, 5, 5, 10, 2, XCfg<Rad<5, 5, 10>, 2>::THREADS, XCfg<Rad<5, 5, 10>, 2>::SMEM_BYTES, launch_x_250_1},
    {252, 0, 7, 6, 6, 2, XCfg<Rad<7, 6, 6>, 2>::THREADS, XCfg<Rad<7, 6, 6>, 2>::SMEM_BYTES, launch_x_252_0},
    {252, 1, 6, 6, 7, 2, XCfg<Rad<6, 6, 7>, 2>::THREADS, XCfg<Rad<6, 6, 7>, 2>::SMEM_BYTES, launch_x_252_1},
    {256, 0, 16, 16, 1, 4, XCfg<Rad<16, 16, 1>, 4>::THREADS, XCfg<Rad<16, 16, 1>, 4>::SMEM_BYTES, launch_x_256_0},
    {270, 0, 9, 5, 6, 2, XCfg<Rad<9, 5, 6>, 2>::THREADS, XCfg<Rad<9, 5, 6>, 2>::SMEM_BYTES, launch_x_270_0},
    {270, 1, 6, 5, 9, 2, XCfg<Rad<6, 5, 9>, 2>::THREADS, XCfg<Rad<6, 5, 9>, 2>::SMEM_BYTES, launch_x_270_1},
    {280, 0, 8, 5, 7, 2, XCfg<Rad<8, 5, 7>, 2>::THREADS, XCfg<Rad<8, 5, 7>, 2>::SMEM_BYTES, launch_x_280_0},
    {280, 1, 7, 5, 8, 2, XCfg<Rad<7, 5, 8>, 2>::THREADS, XCfg<Rad<7, 5, 8>, 2>::SMEM_BYTES, launch_x_280_1},
    {288, 0, 8, 6, 6, 2, XCfg<Rad<8, 6, 6>, 2>::THREADS, XCfg<Rad<8, 6, 6>, 2>::SMEM_BYTES, launch_x_288_0},
    {288, 1, 6, 6, 8, 2, XCfg<Rad<6, 6, 8>, 2>::THREADS, XCfg<Rad<6, 6, 8>, 2>::SMEM_BYTES, launch_x_288_1},
    {294, 0, 7, 6, 7, 2, XCfg<Rad<7, 6, 7>, 2>::THREADS, XCfg<Rad<7, 6, 7>, 2>::SMEM_BYTES, launch_x_294_0},
    {294, 1, 6, 7, 7, 2, XCfg<Rad<6, 7, 7>, 2>::THREADS, XCfg<Rad<6, 7, 7>, 2>::SMEM_BYTES, launch_x_294_1},
    {300, 0, 10, 5, 6, 2, XCfg<Rad<10, 5, 6>, 2>::THREADS, XCfg<Rad<10, 5, 6>, 2>::SMEM_BYTES, launch_x_300_0},
    {300, 1, 6, 5, 10, 2, XCfg<Rad<6, 5, 10>, 2>::THREADS, XCfg<Rad<6, 5, 10>, 2>::SMEM_BYTES, launch_x_300_1},
    {315, 0, 9, 5, 7, 2, XCfg<Rad<9, 5, 7>, 2>::THREADS, XCfg<Rad<9, 5, 7>, 2>::SMEM_BYTES, launch_x_315_0},
    {315, 1, 7, 5, 9, 2, XCfg<Rad<7, 5, 9>, 2>::THREADS, XCfg<Rad<7, 5, 9>, 2>::SMEM_BYTES, launch_x_315_1},
    {320, 0, 8, 5, 8, 2, XCfg<Rad<8, 5, 8>, 2>::THREADS, XCfg<Rad<8, 5, 8>, 2>::SMEM_BYTES, launch_x_320_0},
    {320, 1, 5, 8, 8, 2, XCfg<Rad<5, 8, 8>, 2>::THREADS, XCfg<Rad<5, 8, 8>, 2>::SMEM_BYTES, launch_x_320_1},
    {324, 0, 9, 6, 6, 2, XCfg<Rad<9, 6, 6>, 2>::THREADS, XCfg<Rad<9, 6, 6>, 2>::SMEM_BYTES, launch_x_324_0},
    {324, 1, 6, 6, 9, 2, XCfg<Rad<6, 6, 9>, 2>::THREADS, XCfg<Rad<6, 6, 9>, 2>::SMEM_BYTES, launch_x_324_1},
    {336, 0, 8, 6, 7, 2, XCfg<Rad<8, 6, 7>, 2>::THREADS, XCfg<Rad<8, 6, 7>, 2>::SMEM_BYTES, launch_x_336_0},
    {336, 1, 7, 6, 8, 2, XCfg<Rad<7, 6, 8>, 2>::THREADS, XCfg<Rad<7, 6, 8>, 2>::SMEM_BYTES, launch_x_336_1},
    {343, 0, 7, 7, 7, 2, XCfg<Rad<7, 7, 7>, 2>::THREADS, XCfg<Rad<7, 7, 7>, 2>::SMEM_BYTES, launch_x_343_0},
    {350, 0, 10, 5, 7, 2, XCfg<Rad<10, 5, 7>, 2>::THREADS, XCfg<Rad<10, 5, 7>, 2>::SMEM_BYTES, launch_x_350_0},
    {350, 1, 7, 5, 10, 2, XCfg<Rad<7, 5, 10>, 2>::THREADS, XCfg<Rad<7, 5, 10>, 2>::SMEM_BYTES, launch_x_350_1},
    {360, 0, 10, 6, 6, 2, XCfg<Rad<10, 6, 6>, 2>::THREADS, XCfg<Rad<10, 6, 6>, 2>::SMEM_BYTES, launch_x_360_0},
    {360, 1, 6, 6, 10, 2, XCfg<Rad<6, 6, 10>, 2>::THREADS, XCfg<Rad<6, 6, 10>, 2>::SMEM_BYTES, launch_x_360_1},
    {375, 0, 15, 5, 5, 2, XCfg<Rad<15, 5, 5>, 2>::THREADS, XCfg<Rad<15, 5, 5>, 2>::SMEM_BYTES, launch_x_375_0},
    {375, 1, 5, 5, 15, 2, XCfg<Rad<5, 5, 15>, 2>::THREADS, XCfg<Rad<5, 5, 15>, 2>::SMEM_BYTES, launch_x_375_1},
    {378, 0, 9, 6, 7, 2, XCfg<Rad<9, 6, 7>, 2>::THREADS, XCfg<Rad<9, 6, 7>, 2>::SMEM_BYTES, launch_x_378_0},
    {378, 1, 7, 6, 9, 2, XCfg<Rad<7, 6, 9>, 2>::THREADS, XCfg<Rad<7, 6, 9>, 2>::SMEM_BYTES, launch_x_378_1},
    {384, 0, 8, 6, 8, 2, XCfg<Rad<8, 6, 8>, 2>::THREADS, XCfg<Rad<8, 6, 8>, 2>::SMEM_BYTES, launch_x_384_0},
    {384, 1, 6, 8, 8, 2, XCfg<Rad<6, 8, 8>, 2>::THREADS, XCfg<Rad<6, 8, 8>, 2>::SMEM_BYTES, launch_x_384_1},
    {392, 0, 8, 7, 7, 2, XCfg<Rad<8, 7, 7>, 2>::THREADS, XCfg<Rad<8, 7, 7>, 2>::SMEM_BYTES, launch_x_392_0},
    {392, 1, 7, 7, 8, 2, XCfg<Rad<7, 7, 8>, 2>::THREADS, XCfg<Rad<7, 7, 8>, 2>::SMEM_BYTES, launch_x_392_1},
    {400, 0, 10, 5, 8, 2, XCfg<Rad<10, 5, 8>, 2>::THREADS, XCfg<Rad<10, 5, 8>, 2>::SMEM_BYTES, launch_x_400_0},
    {400, 1, 8, 5, 10, 2, XCfg<Rad<8, 5, 10>, 2>::THREADS, XCfg<Rad<8, 5, 10>, 2>::SMEM_BYTES, launch_x_400_1},
    {405, 0, 9, 5, 9, 2, XCfg<Rad<9, 5, 9>, 2>::THREADS, XCfg<Rad<9, 5, 9>, 2>::SMEM_BYTES, launch_x_405_0},
    {405, 1, 5, 9, 9, 2, XCfg<Rad<5, 9, 9>, 2>::THREADS, XCfg<Rad<5, 9, 9>, 2>::SMEM_BYTES, launch_x_405_1},
    {420, 0, 10, 6, 7, 2, XCfg<Rad<10, 6, 7>, 2>::THREADS, XCfg<Rad<10, 6, 7>, 2>::SMEM_BYTES, launch_x_420_0},
    {420, 1, 7, 6, 10, 2, XCfg<Rad<7, 6, 10>, 2>::THREADS, XCfg<Rad<7, 6, 10>, 2>::SMEM_BYTES, launch_x_420_1},
    {432, 0, 9, 6, 8, 2, XCfg<Rad<9, 6, 8>, 2>::THREADS, XCfg<Rad<9, 6, 8>, 2>::SMEM_BYTES, launch_x_432_0},
    {432, 1, 8, 6, 9, 2, XCfg<Rad<8, 6, 9>, 2>::THREADS, XCfg<Rad<8, 6, 9>, 2>::SMEM_BYTES, launch_x_432_1},
    {441, 0, 9, 7, 7, 2, XCfg<Rad<9, 7, 7>, 2>::THREADS, XCfg<Rad<9, 7, 7>, 2>::SMEM_BYTES, launch_x_441_0},
    {441, 1, 7, 7, 9, 2, XCfg<Rad<7, 7, 9>, 2>::THREADS, XCfg<Rad<7, 7, 9>, 2>::SMEM_BYTES, launch_x_441_1},
    {448, 0, 8, 7, 8, 2, XCfg<Rad<8, 7, 8>, 2>::THREADS, XCfg<Rad<8, 7, 8>, 2>::SMEM_BYTES, launch_x_448_0},
    {448, 1, 7, 8, 8, 2, XCfg<Rad<7, 8, 8>, 2>::THREADS, XCfg<Rad<7, 8, 8>, 2>::SMEM_BYTES, launch_x_448_1},
    {450, 0, 10, 5, 9, 2, XCfg<Rad<10, 5, 9>, 2>::THREADS, XCfg<Rad<10, 5, 9>, 2>::SMEM_BYTES, launch_x_450_0},
    {450, 1, 9, 5, 10, 2, XCfg<Rad<9, 5, 10>, 2>::THREADS, XCfg<Rad<9, 5, 10>, 2>::SMEM_BYTES, launch_x_450_1},
    {480, 0, 10, 6, 8, 2, XCfg<Rad<10, 6, 8>, 2>::THREADS, XCfg<Rad<10, 6, 8>, 2>::SMEM_BYTES, launch_x_480_0},
    {480, 1, 8, 6, 10, 2, XCfg<Rad<8, 6, 10>, 2>::THREADS, XCfg<Rad<8, 6, 10>, 2>::SMEM_BYTES, launch_x_480_1},
    {486, 0, 9, 6, 9, 2, XCfg<Rad<9, 6, 9>, 2>::THREADS, XCfg<Rad<9, 6, 9>, 2>::SMEM_BYTES, launch_x_486_0},
    {486, 1, 6, 9, 9, 2, XCfg<Rad<6, 9, 9>, 2>::THREADS, XCfg<Rad<6, 9, 9>, 2>::SMEM_BYTES, launch_x_486_1},
    {490, 0, 10, 7, 7, 2, XCfg<Rad<10, 7, 7>, 2>::THREADS, XCfg<Rad<10, 7, 7>, 2>::SMEM_BYTES, launch_x_490_0},
    {490, 1, 7, 7, 10, 2, XCfg<Rad<7, 7, 10>, 2>::THREADS, XCfg<Rad<7, 7, 10>, 2>::SMEM_BYTES, launch_x_490_1},
    {500, 0, 10, 5, 10, 2, XCfg<Rad<10, 5, 10>, 2>::THREADS, XCfg<Rad<10, 5, 10>, 2>::SMEM_BYTES, launch_x_500_0},
    {500, 1, 5, 10, 10, 2, XCfg<Rad<5, 10, 10>, 2>::THREADS, XCfg<Rad<5, 10, 10>, 2>::SMEM_BYTES, launch_x_500_1},
    {504, 0, 9, 7, 8, 2, XCfg<Rad<9, 7, 8>, 2>::THREADS, XCfg<Rad<9, 7, 8>, 2>::SMEM_BYTES, launch_x_504_0},
    {504, 1, 8, 7, 9, 2, XCfg<Rad<8, 7, 9>, 2>::THREADS, XCfg<Rad<8, 7, 9>, 2>::SMEM_BYTES, launch_x_504_1},
    {512, 0, 8, 8, 8, 2, XCfg<Rad<8, 8, 8>, 2>::THREADS, XCfg<Rad<8, 8, 8>, 2>::SMEM_BYTES, launch_x_512_0},
    {512, 1, 16, 4, 8, 2, XCfg<Rad<16, 4, 8>, 2>::THREADS, XCfg<Rad<16, 4, 8>, 2>::SMEM_BYTES, launch_x_512_1},
    {525, 0, 15, 5, 7, 2, XCfg<Rad<15, 5, 7>, 2>::THREADS, XCfg<Rad<15, 5, 7>, 2>::SMEM_BYTES, launch_x_525_0},
    {525, 1, 7, 5, 15, 2, XCfg<Rad<7, 5, 15>, 2>::THREADS, XCfg<Rad<7, 5, 15>, 2>::SMEM_BYTES, launch_x_525_1},
    {540, 0, 10, 6, 9, 2, XCfg<Rad<10, 6, 9>, 2>::THREADS, XCfg<Rad<10, 6, 9>, 2>::SMEM_BYTES, launch_x_540_0},
    {540, 1, 9, 6, 10, 2, XCfg<Rad<9, 6, 10>, 2>::THREADS, XCfg<Rad<9, 6, 10>, 2>::SMEM_BYTES, launch_x_540_1},
    {560, 0, 10, 7, 8, 2, XCfg<Rad<10, 7, 8>, 2>::THREADS, XCfg<Rad<10, 7, 8>, 2>::SMEM_BYTES, launch_x_560_0},
    {560, 1, 8, 7, 10, 2, XCfg<Rad<8, 7, 10>, 2>::THREADS, XCfg<Rad<8, 7, 10>, 2>::SMEM_BYTES, launch_x_560_1},
    {567, 0, 9, 7, 9, 2, XCfg<Rad<9, 7, 9>, 2>::THREADS, XCfg<Rad<9, 7, 9>, 2>::SMEM_BYTES, launch_x_567_0},
    {567, 1, 7, 9, 9, 2, XCfg<Rad<7, 9, 9>, 2>::THREADS, XCfg<Rad<7, 9, 9>, 2>::SMEM_BYTES, launch_x_567_1},
    {576, 0, 9, 8, 8, 2, XCfg<Rad<9, 8, 8>, 2>::THREADS, XCfg<Rad<9, 8, 8>, 2>::SMEM_BYTES, launch_x_576_0},
    {576, 1, 8, 8, 9, 2, XCfg<Rad<8, 8, 9>, 2>::THREADS, XCfg<Rad<8, 8, 9>, 2>::SMEM_BYTES, launch_x_576_1},
    {588, 0, 12, 7, 7, 2, XCfg<Rad<12, 7, 7>, 2>::THREADS, XCfg<Rad<12, 7, 7>, 2>::SMEM_BYTES, launch_x_588_0},
    {588, 1, 7, 7, 12, 2, XCfg<Rad<7, 7, 12>, 2>::THREADS, XCfg<Rad<7, 7, 12>, 2>::SMEM_BYTES, launch_x_588_1},
    {600, 0, 10, 6, 10, 2, XCfg<Rad<10, 6, 10>, 2>::THREADS, XCfg<Rad<10, 6, 10>, 2>::SMEM_BYTES, launch_x_600_0},
    {600, 1, 6, 10, 10, 2, XCfg<Rad<6, 10, 10>, 2>::THREADS, XCfg<Rad<6, 10, 10>, 2>::SMEM_BYTES, launch_x_600_1},
    {630, 0, 10, 7, 9, 2, XCfg<Rad<10, 7, 9>, 2>::THREADS, XCfg<Rad<10, 7, 9>, 2>::SMEM_BYTES, launch_x_630_0},
    {630, 1, 9, 7, 10, 2, XCfg<Rad<9, 7, 10>, 2>::THREADS, XCfg<Rad<9, 7, 10>, 2>::SMEM_BYTES, launch_x_630_1},
    {640, 0, 10, 8, 8, 2, XCfg<Rad<10, 8, 8>, 2>::THREADS, XCfg<Rad<10, 8, 8>, 2>::SMEM_BYTES, launch_x_640_0},
    {640, 1, 8, 8, 10, 2, XCfg<Rad<8, 8, 10>, 2>::THREADS, XCfg<Rad<8, 8, 10>, 2>::SMEM_BYTES, launch_x_640_1},
    {648, 0, 9, 8, 9, 2, XCfg<Rad<9, 8, 9>, 2>::THREADS, XCfg<Rad<9, 8, 9>, 2>::SMEM_BYTES, launch_x_648_0},
    {648, 1, 8, 9, 9, 2, XCfg<Rad<8, 9, 9>, 2>::THREADS, XCfg<Rad<8, 9, 9>, 2>::SMEM_BYTES, launch_x_648_1},
    {672, 0, 12, 7, 8, 2, XCfg<Rad<12, 7, 8>, 2>::THREADS, XCfg<Rad<12, 7, 8>, 2>::SMEM_BYTES, launch_x_672_0},
    {672, 1, 8, 7, 12, 2, XCfg<Rad<8, 7, 12>, 2>::THREADS, XCfg<Rad<8, 7, 12>, 2>::SMEM_BYTES, launch_x_672_1},
    {675, 0, 15, 5, 9, 2, XCfg<Rad<15, 5, 9>, 2>::THREADS, XCfg<Rad<15, 5, 9>, 2>::SMEM_BYTES, launch_x_675_0},
    {675, 1, 9, 5, 15, 2, XCfg<Rad<9, 5, 15>, 2>::THREADS, XCfg<Rad<9, 5, 15>, 2>::SMEM_BYTES, launch_x_675_1},
    {686, 0, 14, 7, 7, 2, XCfg<Rad<14, 7, 7>, 2>::THREADS, XCfg<Rad<14, 7, 7>, 2>::SMEM_BYTES, launch_x_686_0},
    {686, 1, 7, 7, 14, 2, XCfg<Rad<7, 7, 14>, 2>::THREADS, XCfg<Rad<7, 7, 14>, 2>::SMEM_BYTES, launch_x_686_1},
    {700, 0, 10, 7, 10, 2, XCfg<Rad<10, 7, 10>, 2>::THREADS, XCfg<Rad<10, 7, 10>, 2>::SMEM_BYTES, launch_x_700_0},
    {700, 1, 7, 10, 10, 2, XCfg<Rad<7, 10, 10>, 2>::THREADS, XCfg<Rad<7, 10, 10>, 2>::SMEM_BYTES, launch_x_700_1},
    {720, 0, 10, 8, 9, 2, XCfg<Rad<10, 8, 9>, 2>::THREADS, XCfg<Rad<10, 8, 9>, 2>::SMEM_BYTES, launch_x_720_0},
    {720, 1, 9, 8, 10, 2, XCfg<Rad<9, 8, 10>, 2>::THREADS, XCfg<Rad<9, 8, 10>, 2>::SMEM_BYTES, launch_x_720_1},
    {729, 0, 9, 9, 9, 2, XCfg<Rad<9, 9, 9>, 2>::THREADS, XCfg<Rad<9, 9, 9>, 2>::SMEM_BYTES, launch_x_729_0},
    {735, 0, 15, 7, 7, 2, XCfg<Rad<15, 7, 7>, 2>::THREADS, XCfg<Rad<15, 7, 7>, 2>::SMEM_BYTES, launch_x_735_0},
    {735, 1, 7, 7, 15, 2, XCfg<Rad<7, 7, 15>, 2>::THREADS, XCfg<Rad<7, 7, 15>, 2>::SMEM_BYTES, launch_x_735_1},
    {750, 0, 15, 5, 10, 2, XCfg<Rad<15, 5, 10>, 2>::THREADS, XCfg<Rad<15, 5, 10>, 2>::SMEM_BYTES, launch_x_750_0},
    {750, 1, 10, 5, 15, 2, XCfg<Rad<10, 5, 15>, 2>::THREADS, XCfg<Rad<10, 5, 15>, 2>::SMEM_BYTES, launch_x_750_1},
    {756, 0, 12, 7, 9, 2, XCfg<Rad<12, 7, 9>, 2>::THREADS, XCfg<Rad<12, 7, 9>, 2>::SMEM_BYTES, launch_x_756_0},
    {756, 1, 9, 7, 12, 2, XCfg<Rad<9, 7, 12>, 2>::THREADS, XCfg<Rad<9, 7, 12>, 2>::SMEM_BYTES, launch_x_756_1},
    {768, 0, 12, 8, 8, 2, XCfg<Rad<12, 8, 8>, 2>::THREADS, XCfg<Rad<12, 8, 8>, 2>::SMEM_BYTES, launch_x_768_0},
    {768, 1, 8, 8, 12, 2, XCfg<Rad<8, 8, 12>, 2>::THREADS, XCfg<Rad<8, 8, 12>, 2>::SMEM_BYTES, launch_x_768_1},
    {784, 0, 14, 7, 8, 2, XCfg<Rad<14, 7, 8>, 2>::THREADS, XCfg<Rad<14, 7, 8>, 2>::SMEM_BYTES, launch_x_784_0},
    {784, 1, 8, 7, 14, 2, XCfg<Rad<8, 7, 14>, 2>::THREADS, XCfg<Rad<8, 7, 14>, 2>::SMEM_BYTES, launch_x_784_1},
    {800, 0, 10, 8, 10, 2, XCfg<Rad<10, 8, 10>, 2>::THREADS, XCfg<Rad<10, 8, 10>, 2>::SMEM_BYTES, launch_x_800_0},
    {800, 1, 8, 10, 10, 2, XCfg<Rad<8, 10, 10>, 2>::THREADS, XCfg<Rad<8, 10, 10>, 2>::SMEM_BYTES, launch_x_800_1},
    {810, 0, 10, 9, 9, 2, XCfg<Rad<10, 9, 9>, 2>::THREADS, XCfg<Rad<10, 9, 9>, 2>::SMEM_BYTES, launch_x_810_0},
    {810, 1, 9, 9, 10, 2, XCfg<Rad<9, 9, 10>, 2>::THREADS, XCfg<Rad<9, 9, 10>, 2>::SMEM_BYTES, launch_x_810_1},
    {840, 0, 12, 7, 10, 2, XCfg<Rad<12, 7, 10>, 2>::THREADS, XCfg<Rad<12, 7, 10>, 2>::SMEM_BYTES, launch_x_840_0},
    {840, 1, 10, 7, 12, 2, XCfg<Rad<10, 7, 12>, 2>::THREADS, XCfg<Rad<10, 7, 12>, 2>::SMEM_BYTES, launch_x_840_1},
    {864, 0, 12, 8, 9, 2, XCfg<Rad<12, 8, 9>, 2>::THREADS, XCfg<Rad<12, 8, 9>, 2>::SMEM_BYTES, launch_x_864_0},
    {864, 1, 9, 8, 12, 2, XCfg<Rad<9, 8, 12>, 2>::THREADS, XCfg<Rad<9, 8, 12>, 2>::SMEM_BYTES, launch_x_864_1},
    {882, 0, 14, 7, 9, 2, XCfg<Rad<14, 7, 9>, 2>::THREADS, XCfg<Rad<14, 7, 9>, 2>::SMEM_BYTES, launch_x_882_0},
    {882, 1, 9, 7, 14, 2, XCfg<Rad<9, 7, 14>, 2>::THREADS, XCfg<Rad<9, 7, 14>, 2>::SMEM_BYTES, launch_x_882_1},
    {896, 0, 14, 8, 8, 2, XCfg<Rad<14, 8, 8>, 2>::THREADS, XCfg<Rad<14, 8, 8>, 2>::SMEM_BYTES, launch_x_896_0},
    {896, 1, 8, 8, 14, 2, XCfg<Rad<8, 8, 14>, 2>::THREADS, XCfg<Rad<8, 8, 14>, 2>::SMEM_BYTES, launch_x_896_1},
    {900, 0, 10, 9, 10, 2, XCfg<Rad<10, 9, 10>, 2>::THREADS, XCfg<Rad<10, 9, 10>, 2>::SMEM_BYTES, launch_x_900_0},
    {900, 1, 9, 10, 10, 2, XCfg<Rad<9, 10, 10>, 2>::THREADS, XCfg<Rad<9, 10, 10>, 2>::SMEM_BYTES, launch_x_900_1},
    {945, 0, 15, 7, 9, 2, XCfg<Rad<15, 7, 9>, 2>::THREADS, XCfg<Rad<15, 7, 9>, 2>::SMEM_BYTES, launch_x_945_0},
    {945, 1, 9, 7, 15, 2, XCfg<Rad<9, 7, 15>, 2>::THREADS, XCfg<Rad<9, 7, 15>, 2>::SMEM_BYTES, launch_x_945_1},
    {960, 0, 12, 8, 10, 2, XCfg<Rad<12, 8, 10>, 2>::THREADS, XCfg<Rad<12, 8, 10>, 2>::SMEM_BYTES, launch_x_960_0},
    {960, 1, 10, 8, 12, 2, XCfg<Rad<10, 8, 12>, 2>::THREADS, XCfg<Rad<10, 8, 12>, 2>::SMEM_BYTES, launch_x_960_1},
    {972, 0, 12, 9, 9, 2, XCfg<Rad<12, 9, 9>, 2>::THREADS, XCfg<Rad<12, 9, 9>, 2>::SMEM_BYTES, launch_x_972_0},
    {972, 1, 9, 9, 12, 2, XCfg<Rad<9, 9, 12>, 2>::THREADS, XCfg<Rad<9, 9, 12>, 2>::SMEM_BYTES, launch_x_972_1},
    {980, 0, 14, 7, 10, 2, XCfg<Rad<14, 7, 10>, 2>::THREADS, XCfg<Rad<14, 7, 10>, 2>::SMEM_BYTES, launch_x_980_0},
    {980, 1, 10, 7, 14, 2, XCfg<Rad<10, 7, 14>, 2>::THREADS, XCfg<Rad<10, 7, 14>, 2>::SMEM_BYTES, launch_x_980_1},
    {1000, 0, 10, 10, 10, 2, XCfg<Rad<10, 10, 10>, 2>::THREADS, XCfg<Rad<10, 10, 10>, 2>::SMEM_BYTES, launch_x_1000_0},
    {1008, 0, 14, 8, 9, 2, XCfg<Rad<14, 8, 9>, 2>::THREADS, XCfg<Rad<14, 8, 9>, 2>::SMEM_BYTES, launch_x_1008_0},
    {1008, 1, 9, 8, 14, 2, XCfg<Rad<9, 8, 14>, 2>::THREADS, XCfg<Rad<9, 8, 14>, 2>::SMEM_BYTES, launch_x_1008_1},
    {1024, 0, 16, 8, 8, 2, XCfg<Rad<16, 8, 8>, 2>::THREADS, XCfg<Rad<16, 8, 8>, 2>::SMEM_BYTES, launch_x_1024_0},
    {1024, 1, 8, 8, 16, 2, XCfg<Rad<8, 8, 16>, 2>::THREADS, XCfg<Rad<8, 8, 16>, 2>::SMEM_BYTES, launch_x_1024_1},
    {1050, 0, 15, 7, 10, 2, XCfg<Rad<15, 7, 10>, 2>::THREADS, XCfg<Rad<15, 7, 10>, 2>::SMEM_BYTES, launch_x_1050_0},
    {1050, 1, 10, 7, 15, 2, XCfg<Rad<10, 7, 15>, 2>::THREADS, XCfg<Rad<10, 7, 15>, 2>::SMEM_BYTES, launch_x_1050_1},
    {1080, 0, 12, 9, 10, 2, XCfg<Rad<12, 9, 10>, 2>::THREADS, XCfg<Rad<12, 9, 10>, 2>::SMEM_BYTES, launch_x_1080_0},
    {1080, 1, 10, 9, 12, 2, XCfg<Rad<10, 9, 12>, 2>::THREADS, XCfg<Rad<10, 9, 12>, 2>::SMEM_BYTES, launch_x_1080_1},
    {1120, 0, 14, 8, 10, 2, XCfg<Rad<14, 8, 10>, 2>::THREADS, XCfg<Rad<14, 8, 10>, 2>::SMEM_BYTES, launch_x_1120_0},
    {1120, 1, 10, 8, 14, 2, XCfg<Rad<10, 8, 14>, 2>::THREADS, XCfg<Rad<10, 8, 14>, 2>::SMEM_BYTES, launch_x_1120_1},
    {1125, 0, 15, 5, 15, 1, XCfg<Rad<15, 5, 15>, 1>::THREADS, XCfg<Rad<15, 5, 15>, 1>::SMEM_BYTES, launch_x_1125_0},
    {1125, 1, 5, 15, 15, 1, XCfg<Rad<5, 15, 15>, 1>::THREADS, XCfg<Rad<5, 15, 15>, 1>::SMEM_BYTES, launch_x_1125_1},
    {1134, 0, 14, 9, 9, 2, XCfg<Rad<14, 9, 9>, 2>::THREADS, XCfg<Rad<14, 9, 9>, 2>::SMEM_BYTES, launch_x_1134_0},
    {1134, 1, 9, 9, 14, 2, XCfg<Rad<9, 9, 14>, 2>::THREADS, XCfg<Rad<9, 9, 14>, 2>::SMEM_BYTES, launch_x_1134_1},
    {1152, 0, 12, 8, 12, 1, XCfg<Rad<12, 8, 12>, 1>::THREADS, XCfg<Rad<12, 8, 12>, 1>::SMEM_BYTES, launch_x_1152_0},
    {1152, 1, 8, 12, 12, 1, XCfg<Rad<8, 12, 12>, 1>::THREADS, XCfg<Rad<8, 12, 12>, 1>::SMEM_BYTES, launch_x_1152_1},
    {1176, 0, 14, 7, 12, 1, XCfg<Rad<14, 7, 12>, 1>::THREADS, XCfg<Rad<14, 7, 12>, 1>::SMEM_BYTES, launch_x_1176_0},
    {1176, 1, 12, 7, 14, 1, XCfg<Rad<12, 7, 14>, 1>::THREADS, XCfg<Rad<12, 7, 14>, 1>::SMEM_BYTES, launch_x_1176_1},
    {1200, 0, 12, 10, 10, 1, XCfg<Rad<12, 10, 10>, 1>::THREADS, XCfg<Rad<12, 10, 10>, 1>::SMEM_BYTES, launch_x_1200_0},
    {1200, 1, 10, 10, 12, 1, XCfg<Rad<10, 10, 12>, 1>::THREADS, XCfg<Rad<10, 10, 12>, 1>::SMEM_BYTES, launch_x_1200_1},
    {1215, 0, 15, 9, 9, 1, XCfg<Rad<15, 9, 9>, 1>::THREADS, XCfg<Rad<15, 9, 9>, 1>::SMEM_BYTES, launch_x_1215_0},
    {1215, 1, 9, 9, 15, 1, XCfg<Rad<9, 9, 15>, 1>::THREADS, XCfg<Rad<9, 9, 15>, 1>::SMEM_BYTES, launch_x_1215_1},
    {1260, 0, 14, 9, 10, 1, XCfg<Rad<14, 9, 10>, 1>::THREADS, XCfg<Rad<14, 9, 10>, 1>::SMEM_BYTES, launch_x_1260_0},
    {1260, 1, 10, 9, 14, 1, XCfg<Rad<10, 9, 14>, 1>::THREADS, XCfg<Rad<10, 9, 14>, 1>::SMEM_BYTES, launch_x_1260_1},
    {1280, 0, 16, 8, 10, 1, XCfg<Rad<16, 8, 10>, 1>::THREADS, XCfg<Rad<16, 8, 10>, 1>::SMEM_BYTES, launch_x_1280_0},
    {1280, 1, 10, 8, 16, 1, XCfg<Rad<10, 8, 16>, 1>::THREADS, XCfg<Rad<10, 8, 16>, 1>::SMEM_BYTES, launch_x_1280_1},
    {1296, 0, 12, 9, 12, 1, XCfg<Rad<12, 9, 12>, 1>::THREADS, XCfg<Rad<12, 9, 12>, 1>::SMEM_BYTES, launch_x_1296_0},
    {1296, 1, 9, 12, 12, 1, XCfg<Rad<9, 12, 12>, 1>::THREADS, XCfg<Rad<9, 12, 12>, 1>::SMEM_BYTES, launch_x_1296_1},
    {1344, 0, 14, 8, 12, 1, XCfg<Rad<14, 8, 12>, 1>::THREADS, XCfg<Rad<14, 8, 12>, 1>::SMEM_BYTES, launch_x_1344_0},
    {1344, 1, 12, 8, 14, 1, XCfg<Rad<12, 8, 14>, 1>::THREADS, XCfg<Rad<12, 8, 14>, 1>::SMEM_BYTES, launch_x_1344_1},
    {1350, 0, 15, 9, 10, 1, XCfg<Rad<15, 9, 10>, 1>::THREADS, XCfg<Rad<15, 9, 10>, 1>::SMEM_BYTES, launch_x_1350_0},
    {1350, 1, 10, 9, 15, 1, XCfg<Rad<10, 9, 15>, 1>::THREADS, XCfg<Rad<10, 9, 15>, 1>::SMEM_BYTES, launch_x_1350_1},
    {1372, 0, 14, 7, 14, 1, XCfg<Rad<14, 7, 14>, 1>::THREADS, XCfg<Rad<14, 7, 14>, 1>::SMEM_BYTES, launch_x_1372_0},
    {1372, 1, 7, 14, 14, 1, XCfg<Rad<7, 14, 14>, 1>::THREADS, XCfg<Rad<7, 14, 14>, 1>::SMEM_BYTES, launch_x_1372_1},
    {1400, 0, 14, 10, 10, 1, XCfg<Rad<14, 10, 10>, 1>::THREADS, XCfg<Rad<14, 10, 10>, 1>::SMEM_BYTES, launch_x_1400_0},
    {1400, 1, 10, 10, 14, 1, XCfg<Rad<10, 10, 14>, 1>::THREADS, XCfg<Rad<10, 10, 14>, 1>::SMEM_BYTES, launch_x_1400_1},
    {1440, 0, 12, 10, 12, 1, XCfg<Rad<12, 10, 12>, 1>::THREADS, XCfg<Rad<12, 10, 12>, 1>::SMEM_BYTES, launch_x_1440_0},
    {1440, 1, 10, 12, 12, 1, XCfg<Rad<10, 12, 12>, 1>::THREADS, XCfg<Rad<10, 12, 12>, 1>::SMEM_BYTES, launch_x_1440_1},
    {1470, 0, 15, 7, 14, 1, XCfg<Rad<15, 7, 14>, 1>::THREADS, XCfg<Rad<15, 7, 14>, 1>::SMEM_BYTES, launch_x_1470_0},
    {1470, 1, 14, 7, 15, 1, XCfg<Rad<14, 7, 15>, 1>::THREADS, XCfg<Rad<14, 7, 15>, 1>::SMEM_BYTES, launch_x_1470_1},
    {1500, 0, 15, 10, 10, 1, XCfg<Rad<15, 10, 10>, 1>::THREADS, XCfg<Rad<15, 10, 10>, 1>::SMEM_BYTES, launch_x_1500_0},
    {1500, 1, 10, 10, 15, 1, XCfg<Rad<10, 10, 15>, 1>::THREADS, XCfg<Rad<10, 10, 15>, 1>::SMEM_BYTES, launch_x_1500_1},
    {1512, 0, 14, 9, 12, 1, XCfg<Rad<14, 9, 12>, 1>::THREADS, XCfg<Rad<14, 9, 12>, 1>::SMEM_BYTES, launch_x_1512_0},
    {1512, 1, 12, 9, 14, 1, XCfg<Rad<12, 9, 14>, 1>::THREADS, XCfg<Rad<12, 9, 14>, 1>::SMEM_BYTES, launch_x_1512_1},
    {1536, 0, 16, 8, 12, 1, XCfg<Rad<16, 8, 12>, 1>::THREADS, XCfg<Rad<16, 8, 12>, 1>::SMEM_BYTES, launch_x_1536_0},
    {1536, 1, 12, 8, 16, 1, XCfg<Rad<12, 8, 16>, 1>::THREADS, XCfg<Rad<12, 8, 16>, 1>::SMEM_BYTES, launch_x_1536_1},
    {1568, 0, 14, 8, 14, 1, XCfg<Rad<14, 8, 14>, 1>::THREADS, XCfg<Rad<14, 8, 14>, 1>::SMEM_BYTES, launch_x_1568_0},
    {1568, 1, 8, 14, 14, 1, XCfg<Rad<8, 14, 14>, 1>::THREADS, XCfg<Rad<8, 14, 14>, 1>::SMEM_BYTES, launch_x_1568_1},
    {1575, 0, 15, 7, 15, 1, XCfg<Rad<15, 7, 15>, 1>::THREADS, XCfg<Rad<15, 7, 15>, 1>::SMEM_BYTES, launch_x_1575_0},
    {1575, 1, 7, 15, 15, 1, XCfg<Rad<7, 15, 15>, 1>::THREADS, XCfg<Rad<7, 15, 15>, 1>::SMEM_BYTES, launch_x_1575_1},
    {1600, 0, 16, 10, 10, 1, XCfg<Rad<16, 10, 10>, 1>::THREADS, XCfg<Rad<16, 10, 10>, 1>::SMEM_BYTES, launch_x_1600_0},
    {1600, 1, 10, 10, 16, 1, XCfg<Rad<10, 10, 16>, 1>::THREADS, XCfg<Rad<10, 10, 16>, 1>::SMEM_BYTES, launch_x_1600_1},
    {1620, 0, 15, 9, 12, 1, XCfg<Rad<15, 9, 12>, 1>::THREADS, XCfg<Rad<15, 9, 12>, 1>::SMEM_BYTES, launch_x_1620_0},
    {1620, 1, 12, 9, 15, 1, XCfg<Rad<12, 9, 15>, 1>::THREADS, XCfg<Rad<12, 9, 15>, 1>::SMEM_BYTES, launch_x_1620_1},
    {1680, 0, 14, 10, 12, 1, XCfg<Rad<14, 10, 12>, 1>::THREADS, XCfg<Rad<14, 10, 12>, 1>::SMEM_BYTES, launch_x_1680_0},
    {1680, 1, 12, 10, 14, 1, XCfg<Rad<12, 10, 14>, 1>::THREADS, XCfg<Rad<12, 10, 14>, 1>::SMEM_BYTES, launch_x_1680_1},
    {1728, 0, 12, 12, 12, 1, XCfg<Rad<12, 12, 12>, 1>::THREADS, XCfg<Rad<12, 12, 12>, 1>::SMEM_BYTES, launch_x_1728_0},
    {1728, 1, 16, 9, 12, 1, XCfg<Rad<16, 9, 12>, 1>::THREADS, XCfg<Rad<16, 9, 12>, 1>::SMEM_BYTES, launch_x_1728_1},
    {1764, 0, 14, 9, 14, 1, XCfg<Rad<14, 9, 14>, 1>::THREADS, XCfg<Rad<14, 9, 14>, 1>::SMEM_BYTES, launch_x_1764_0},
    {1764, 1, 9, 14, 14, 1, XCfg<Rad<9, 14, 14>, 1>::THREADS, XCfg<Rad<9, 14, 14>, 1>::SMEM_BYTES, launch_x_1764_1},
    {1792, 0, 16, 8, 14, 1, XCfg<Rad<16, 8, 14>, 1>::THREADS, XCfg<Rad<16, 8, 14>, 1>::SMEM_BYTES, launch_x_1792_0},
    {1792, 1, 14, 8, 16, 1, XCfg<Rad<14, 8, 16>, 1>::THREADS, XCfg<Rad<14, 8, 16>, 1>::SMEM_BYTES, launch_x_1792_1},
    {1800, 0, 15, 10, 12, 1, XCfg<Rad<15, 10, 12>, 1>::THREADS, XCfg<Rad<15, 10, 12>, 1>::SMEM_BYTES, launch_x_1800_0},
    {1800, 1, 12, 10, 15, 1, XCfg<Rad<12, 10, 15>, 1>::THREADS, XCfg<Rad<12, 10, 15>, 1>::SMEM_BYTES, launch_x_1800_1},
    {1890, 0, 15, 9, 14, 1, XCfg<Rad<15, 9, 14>, 1>::THREADS, XCfg<Rad<15, 9, 14>, 1>::SMEM_BYTES, launch_x_1890_0},
    {1890, 1, 14, 9, 15, 1, XCfg<Rad<14, 9, 15>, 1>::THREADS, XCfg<Rad<14, 9, 15>, 1>::SMEM_BYTES, launch_x_1890_1},
    {1920, 0, 16, 10, 12, 1, XCfg<Rad<16, 10, 12>, 1>::THREADS, XCfg<Rad<16, 10, 12>, 1>::SMEM_BYTES, launch_x_1920_0},
    {1920, 1, 12, 10, 16, 1, XCfg<Rad<12, 10, 16>, 1>::THREADS, XCfg<Rad<12, 10, 16>, 1>::SMEM_BYTES, launch_x_1920_1},
    {1960, 0, 14, 10, 14, 1, XCfg<Rad<14, 10, 14>, 1>::THREADS, XCfg<Rad<14, 10, 14>, 1>::SMEM_BYTES, launch_x_1960_0},
    {1960, 1, 10, 14, 14, 1, XCfg<Rad<10, 14, 14>, 1>::THREADS, XCfg<Rad<10, 14, 14>, 1>::SMEM_BYTES, launch_x_1960_1},
    {2016, 0, 14, 12, 12, 1, XCfg<Rad<14, 12, 12>, 1>::THREADS, XCfg<Rad<14, 12, 12>, 1>::SMEM_BYTES, launch_x_2016_0},
    {2016, 1, 12, 12, 14, 1, XCfg<Rad<12, 12, 14>, 1>::THREADS, XCfg<Rad<12, 12, 14>, 1>::SMEM_BYTES, launch_x_2016_1},
    {2025, 0, 15, 9, 15, 1, XCfg<Rad<15, 9, 15>, 1>::THREADS, XCfg<Rad<15, 9, 15>, 1>::SMEM_BYTES, launch_x_2025_0},
    {2025, 1, 9, 15, 15, 1, XCfg<Rad<9, 15, 15>, 1>::THREADS, XCfg<Rad<9, 15, 15>, 1>::SMEM_BYTES, launch_x_2025_1},
    {2048, 0, 16, 8, 16, 1, XCfg<Rad<16, 8, 16>, 1>::THREADS, XCfg<Rad<16, 8, 16>, 1>::SMEM_BYTES, launch_x_2048_0},
    {2048, 1, 8, 16, 16, 1, XCfg<Rad<8, 16, 16>, 1>::THREADS, XCfg<Rad<8, 16, 16>, 1>::SMEM_BYTES, launch_x_2048_1},
};
static const YPlan kYPlans[] = {
    {2, 0, 2, 1, 1, YCfg<Rad<2, 1, 1>>::THREADS, YCfg<Rad<2, 1, 1>>::SMEM_BYTES, launch_y_2_0},
    {3, 0, 3, 1, 1, YCfg<Rad<3, 1, 1>>::THREADS, YCfg<Rad<3, 1, 1>>::SMEM_BYTES, launch_y_3_0},
    {4, 0, 2, 2, 1, YCfg<Rad<2, 2, 1>>::THREADS, YCfg<Rad<2, 2, 1>>::SMEM_BYTES, launch_y_4_0},
    {4, 1, 4, 1, 1, YCfg<Rad<4, 1, 1>>::THREADS, YCfg<Rad<4, 1, 1>>::SMEM_BYTES, launch_y_4_1},
    {5, 0, 5, 1, 1, YCfg<Rad<5, 1, 1>>::THREADS, YCfg<Rad<5, 1, 1>>::SMEM_BYTES, launch_y_5_0},
    {6, 0, 3, 2, 1, YCfg<Rad<3, 2, 1>>::THREADS, YCfg<Rad<3, 2, 1>>::SMEM_BYTES, launch_y_6_0},
    {6, 1, 2, 3, 1, YCfg<Rad<2, 3, 1>>::THREADS, YCfg<Rad<2, 3, 1>>::SMEM_BYTES, launch_y_6_1},
    {6, 2, 6, 1, 1, YCfg<Rad<6, 1, 1>>::THREADS, YCfg<Rad<6, 1, 1>>::SMEM_BYTES, launch_y_6_2},
    {7, 0, 7, 1, 1, YCfg<Rad<7, 1, 1>>::THREADS, YCfg<Rad<7, 1, 1>>::SMEM_BYTES, launch_y_7_0},
    {8, 0, 4, 2, 1, YCfg<Rad<4, 2, 1>>::THREADS, YCfg<Rad<4, 2, 1>>::SMEM_BYTES, launch_y_8_0},
    {8, 1, 2, 4, 1, YCfg<Rad<2, 4, 1>>::THREADS, YCfg<Rad<2, 4, 1>>::SMEM_BYTES, launch_y_8_1},
    {8, 2, 8, 1, 1, YCfg<Rad<8, 1, 1>>::THREADS, YCfg<Rad<8, 1, 1>>::SMEM_BYTES, launch_y_8_2},
    {9, 0, 3, 3, 1, YCfg<Rad<3, 3, 1>>::THREADS, YCfg<Rad<3, 3, 1>>::SMEM_BYTES, launch_y_9_0},
    {9, 1, 9, 1, 1, YCfg<Rad<9, 1, 1>>::THREADS, YCfg<Rad<9, 1, 1>>::SMEM_BYTES, launch_y_9_1},
    {10, 0, 5, 2, 1, YCfg<Rad<5, 2, 1>>::THREADS, YCfg<Rad<5, 2, 1>>::SMEM_BYTES, launch_y_10_0},
    {10, 1, 2, 5, 1, YCfg<Rad<2, 5, 1>>::THREADS, YCfg<Rad<2, 5, 1>>::SMEM_BYTES, launch_y_10_1},
    {10, 2, 10, 1, 1, YCfg<Rad<10, 1, 1>>::THREADS, YCfg<Rad<10, 1, 1>>::SMEM_BYTES, launch_y_10_2},
    {12, 0, 4, 3, 1, YCfg<Rad<4, 3, 1>>::THREADS, YCfg<Rad<4, 3, 1>>::SMEM_BYTES, launch_y_12_0},
    {12, 1, 3, 4, 1, YCfg<Rad<3, 4, 1>>::THREADS, YCfg<Rad<3, 4, 1>>::SMEM_BYTES, launch_y_12_1},
    {12, 2, 6, 2, 1, YCfg<Rad<6, 2, 1>>::THREADS, YCfg<Rad<6, 2, 1>>::SMEM_BYTES, launch_y_12_2},
    {14, 0, 7, 2, 1, YCfg<Rad<7, 2, 1>>::THREADS, YCfg<Rad<7, 2, 1>>::SMEM_BYTES, launch_y_14_0},
    {14, 1, 2, 7, 1, YCfg<Rad<2, 7, 1>>::THREADS, YCfg<Rad<2, 7, 1>>::SMEM_BYTES, launch_y_14_1},
    {14, 2, 14, 1, 1, YCfg<Rad<14, 1, 1>>::THREADS, YCfg<Rad<14, 1, 1>>::SMEM_BYTES, launch_y_14_2},
    {15, 0, 5, 3, 1, YCfg<Rad<5, 3, 1>>::THREADS, YCfg<Rad<5, 3, 1>>::SMEM_BYTES, launch_y_15_0},
    {15, 1, 3, 5, 1, YCfg<Rad<3, 5, 1>>::THREADS, YCfg<Rad<3, 5, 1>>::SMEM_BYTES, launch_y_15_1},
    {15, 2, 15, 1, 1, YCfg<Rad<15, 1, 1>>::THREADS, YCfg<Rad<15, 1, 1>>::SMEM_BYTES, launch_y_15_2},
    {16, 0, 4, 4, 1, YCfg<Rad<4, 4, 1>>::THREADS, YCfg<Rad<4, 4, 1>>::SMEM_BYTES, launch_y_16_0},
    {16, 1, 8, 2, 1, YCfg<Rad<8, 2, 1>>::THREADS, YCfg<Rad<8, 2, 1>>::SMEM_BYTES, launch_y_16_1},
    {16, 2, 2, 8, 1, YCfg<Rad<2, 8, 1>>::THREADS, YCfg<Rad<2, 8, 1>>::SMEM_BYTES, launch_y_16_2},
    {18, 0, 6, 3, 1, YCfg<Rad<6, 3, 1>>::THREADS, YCfg<Rad<6, 3, 1>>::SMEM_BYTES, launch_y_18_0},
    {18, 1, 3, 6, 1, YCfg<Rad<3, 6, 1>>::THREADS, YCfg<Rad<3, 6, 1>>::SMEM_BYTES, launch_y_18_1},
    {18, 2, 9, 2, 1, YCfg<Rad<9, 2, 1>>::THREADS, YCfg<Rad<9, 2, 1>>::SMEM_BYTES, launch_y_18_2},
    {20, 0, 5, 4, 1, YCfg<Rad<5, 4, 1>>::THREADS, YCfg<Rad<5, 4, 1>>::SMEM_BYTES, launch_y_20_0},
    {20, 1, 4, 5, 1, YCfg<Rad<4, 5, 1>>::THREADS, YCfg<Rad<4, 5, 1>>::SMEM_BYTES, launch_y_20_1},
    {20, 2, 10, 2, 1, YCfg<Rad<10, 2, 1>>::THREADS, YCfg<Rad<10, 2, 1>>::SMEM_BYTES, launch_y_20_2},
    {21, 0, 7, 3, 1, YCfg<Rad<7, 3, 1>>::THREADS, YCfg<Rad<7, 3, 1>>::SMEM_BYTES, launch_y_21_0},
    {21, 1, 3, 7, 1, YCfg<Rad<3, 7, 1>>::THREADS, YCfg<Rad<3, 7, 1>>::SMEM_BYTES, launch_y_21_1},
    {24, 0, 6, 4, 1, YCfg<Rad<6, 4, 1>>::THREADS, YCfg<Rad<6, 4, 1>>::SMEM_BYTES, launch_y_24_0},
    {24, 1, 4, 6, 1, YCfg<Rad<4, 6, 1>>::THREADS, YCfg<Rad<4, 6, 1>>::SMEM_BYTES, launch_y_24_1},
    {24, 2, 8, 3, 1, YCfg<Rad<8, 3, 1>>::THREADS, YCfg<Rad<8, 3, 1>>::SMEM_BYTES, launch_y_24_2},
    {25, 0, 5, 5, 1, YCfg<Rad<5, 5, 1>>::THREADS, YCfg<Rad<5, 5, 1>>::SMEM_BYTES, launch_y_25_0},
    {27, 0, 9, 3, 1, YCfg<Rad<9, 3, 1>>::THREADS, YCfg<Rad<9, 3, 1>>::SMEM_BYTES, launch_y_27_0},
    {27, 1, 3, 9, 1, YCfg<Rad<3, 9, 1>>::THREADS, YCfg<Rad<3, 9, 1>>::SMEM_BYTES, launch_y_27_1},
    {28, 0, 7, 4, 1, YCfg<Rad<7, 4, 1>>::THREADS, YCfg<Rad<7, 4, 1>>::SMEM_BYTES, launch_y_28_0},
    {28, 1, 4, 7, 1, YCfg<Rad<4, 7, 1>>::THREADS, YCfg<Rad<4, 7, 1>>::SMEM_BYTES, launch_y_28_1},
    {28, 2, 14, 2, 1, YCfg<Rad<14, 2, 1>>::THREADS, YCfg<Rad<14, 2, 1>>::SMEM_BYTES, launch_y_28_2},
    {30, 0, 6, 5, 1, YCfg<Rad<6, 5, 1>>::THREADS, YCfg<Rad<6, 5, 1>>::SMEM_BYTES, launch_y_30_0},
    {30, 1, 5, 6, 1, YCfg<Rad<5, 6, 1>>::THREADS, YCfg<Rad<5, 6, 1>>::SMEM_BYTES, launch_y_30_1},
    {30, 2, 10, 3, 1, YCfg<Rad<10, 3, 1>>::THREADS, YCfg<Rad<10, 3, 1>>::SMEM_BYTES, launch_y_30_2},
    {32, 0, 8, 4, 1, YCfg<Rad<8, 4, 1>>::THREADS, YCfg<Rad<8, 4, 1>>::SMEM_BYTES, launch_y_32_0},
    {32, 1, 4, 8, 1, YCfg<Rad<4, 8, 1>>::THREADS, YCfg<Rad<4, 8, 1>>::SMEM_BYTES, launch_y_32_1},
    {32, 2, 16, 2, 1, YCfg<Rad<16, 2, 1>>::THREADS, YCfg<Rad<16, 2, 1>>::SMEM_BYTES, launch_y_32_2},
    {35, 0, 7, 5, 1, YCfg<Rad<7, 5, 1>>::THREADS, YCfg<Rad<7, 5, 1>>::SMEM_BYTES, launch_y_35_0},
    {35, 1, 5, 7, 1, YCfg<Rad<5, 7, 1>>::THREADS, YCfg<Rad<5, 7, 1>>::SMEM_BYTES, launch_y_35_1},
    {36, 0, 6, 6, 1, YCfg<Rad<6, 6, 1>>::THREADS, YCfg<Rad<6, 6, 1>>::SMEM_BYTES, launch_y_36_0},
    {36, 1, 9, 4, 1, YCfg<Rad<9, 4, 1>>::THREADS, YCfg<Rad<9, 4, 1>>::SMEM_BYTES, launch_y_36_1},
    {36, 2, 4, 9, 1, YCfg<Rad<4, 9, 1>>::THREADS, YCfg<Rad<4, 9, 1>>::SMEM_BYTES, launch_y_36_2},
    {40, 0, 8, 5, 1, YCfg<Rad<8, 5, 1>>::THREADS, YCfg<Rad<8, 5, 1>>::SMEM_BYTES, launch_y_40_0},
    {40, 1, 5, 8, 1, YCfg<Rad<5, 8, 1>>::THREADS, YCfg<Rad<5, 8, 1>>::SMEM_BYTES, launch_y_40_1},
    {40, 2, 10, 4, 1, YCfg<Rad<10, 4, 1>>::THREADS, YCfg<Rad<10, 4, 1>>::SMEM_BYTES, launch_y_40_2},
    {42, 0, 7, 6, 1, YCfg<Rad<7, 6, 1>>::THREADS, YCfg<Rad<7, 6, 1>>::SMEM_BYTES, launch_y_42_0},
    {42, 1, 6, 7, 1, YCfg<Rad<6, 7, 1>>::THREADS, YCfg<Rad<6, 7, 1>>::SMEM_BYTES, launch_y_42_1},
    {42, 2, 14, 3, 1, YCfg<Rad<14, 3, 1>>::THREADS, YCfg<Rad<14, 3, 1>>::SMEM_BYTES, launch_y_42_2},
    {45, 0, 9, 5, 1, YCfg<Rad<9, 5, 1>>::THREADS, YCfg<Rad<9, 5, 1>>::SMEM_BYTES, launch_y_45_0},
    {45, 1, 5, 9, 1, YCfg<Rad<5, 9, 1>>::THREADS, YCfg<Rad<5, 9, 1>>::SMEM_BYTES, launch_y_45_1},
    {45, 2, 15, 3, 1, YCfg<Rad<15, 3, 1>>::THREADS, YCfg<Rad<15, 3, 1>>::SMEM_BYTES, launch_y_45_2},
    {48, 0, 8, 6, 1, YCfg<Rad<8, 6, 1>>::THREADS, YCfg<Rad<8, 6, 1>>::SMEM_BYTES, launch_y_48_0},
    {48, 1, 6, 8, 1, YCfg<Rad<6, 8, 1>>::THREADS, YCfg<Rad<6, 8, 1>>::SMEM_BYTES, launch_y_48_1},
    {48, 2, 12, 4, 1, YCfg<Rad<12, 4, 1>>::THREADS, YCfg<Rad<12, 4, 1>>::SMEM_BYTES, launch_y_48_2},
    {49, 0, 7, 7, 1, YCfg<Rad<7, 7, 1>>::THREADS, YCfg<Rad<7, 7, 1>>::SMEM_BYTES, launch_y_49_0},
    {50, 0, 10, 5, 1, YCfg<Rad<10, 5, 1>>::THREADS, YCfg<Rad<10, 5, 1>>::SMEM_BYTES, launch_y_50_0},
    {50, 1, 5, 10, 1, YCfg<Rad<5, 10, 1>>::THREADS, YCfg<Rad<5, 10, 1>>::SMEM_BYTES, launch_y_50_1},
    {50, 2, 2, 5, 5, YCfg<Rad<2, 5, 5>>::THREADS, YCfg<Rad<2, 5, 5>>::SMEM_BYTES, launch_y_50_2},
    {54, 0, 9, 6, 1, YCfg<Rad<9, 6, 1>>::THREADS, YCfg<Rad<9, 6, 1>>::SMEM_BYTES, launch_y_54_0},
    {54, 1, 6, 9, 1, YCfg<Rad<6, 9, 1>>::THREADS, YCfg<Rad<6, 9, 1>>::SMEM_BYTES, launch_y_54_1},
    {54, 2, 3, 3, 6, YCfg<Rad<3, 3, 6>>::THREADS, YCfg<Rad<3, 3, 6>>::SMEM_BYTES, launch_y_54_2},
    {56, 0, 8, 7, 1, YCfg<Rad<8, 7, 1>>::THREADS, YCfg<Rad<8, 7, 1>>::SMEM_BYTES, launch_y_56_0},
    {56, 1, 7, 8, 1, YCfg<Rad<7, 8, 1>>::THREADS, YCfg<Rad<7, 8, 1>>::SMEM_BYTES, launch_y_56_1},
    {56, 2, 14, 4, 1, YCfg<Rad<14, 4, 1>>::THREADS, YCfg<Rad<14, 4, 1>>::SMEM_BYTES, launch_y_56_2},
    {60, 0, 10, 6, 1, YCfg<Rad<10, 6, 1>>::THREADS, YCfg<Rad<10, 6, 1>>::SMEM_BYTES, launch_y_60_0},
    {60, 1, 6, 10, 1, YCfg<Rad<6, 10, 1>>::THREADS, YCfg<Rad<6, 10, 1>>::SMEM_BYTES, launch_y_60_1},
    {60, 2, 12, 5, 1, YCfg<Rad<12, 5, 1>>::THREADS, YCfg<Rad<12, 5, 1>>::SMEM_BYTES, launch_y_60_2},
    {63, 0, 9, 7, 1, YCfg<Rad<9, 7, 1>>::THREADS, YCfg<Rad<9, 7, 1>>::SMEM_BYTES, launch_y_63_0},
    {63, 1, 7, 9, 1, YCfg<Rad<7, 9, 1>>::THREADS, YCfg<Rad<7, 9, 1>>::SMEM_BYTES, launch_y_63_1},
    {63, 2, 3, 3, 7, YCfg<Rad<3, 3, 7>>::THREADS, YCfg<Rad<3, 3, 7>>::SMEM_BYTES, launch_y_63_2},
    {64, 0, 8, 8, 1, YCfg<Rad<8, 8, 1>>::THREADS, YCfg<Rad<8, 8, 1>>::SMEM_BYTES, launch_y_64_0},
    {64, 1, 16, 4, 1, YCfg<Rad<16, 4, 1>>::THREADS, YCfg<Rad<16, 4, 1>>::SMEM_BYTES, launch_y_64_1},
    {64, 2, 4, 16, 1, YCfg<Rad<4, 16, 1>>::THREADS, YCfg<Rad<4, 16, 1>>::SMEM_BYTES, launch_y_64_2},
    {70, 0, 10, 7, 1, YCfg<Rad<10, 7, 1>>::THREADS, YCfg<Rad<10, 7, 1>>::SMEM_BYTES, launch_y_70_0},
    {70, 1, 7, 10, 1, YCfg<Rad<7, 10, 1>>::THREADS, YCfg<Rad<7, 10, 1>>::SMEM_BYTES, launch_y_70_1},
    {70, 2, 14, 5, 1, YCfg<Rad<14, 5, 1>>::THREADS, YCfg<Rad<14, 5, 1>>::SMEM_BYTES, launch_y_70_2},
    {72, 0, 9, 8, 1, YCfg<Rad<9, 8, 1>>::THREADS, YCfg<Rad<9, 8, 1>>::SMEM_BYTES, launch_y_72_0},
    {72, 1, 8, 9, 1, YCfg<Rad<8, 9, 1>>::THREADS, YCfg<Rad<8, 9, 1>>::SMEM_BYTES, launch_y_72_1},
    {72, 2, 12, 6, 1, YCfg<Rad<12, 6, 1>>::THREADS, YCfg<Rad<12, 6, 1>>::SMEM_BYTES, launch_y_72_2},
    {75, 0, 15, 5, 1, YCfg<Rad<15, 5, 1>>::THREADS, YCfg<Rad<15, 5, 1>>::SMEM_BYTES, launch_y_75_0},
    {75, 1, 5, 15, 1, YCfg<Rad<5, 15, 1>>::THREADS, YCfg<Rad<5, 15, 1>>::SMEM_BYTES, launch_y_75_1},
    {75, 2, 3, 5, 5, YCfg<Rad<3, 5, 5>>::THREADS, YCfg<Rad<3, 5, 5>>::SMEM_BYTES, launch_y_75_2},
    {80, 0, 10, 8, 1, YCfg<Rad<10, 8, 1>>::THREADS, YCfg<Rad<10, 8, 1>>::SMEM_BYTES, launch_y_80_0},
    {80, 1, 8, 10, 1, YCfg<Rad<8, 10, 1>>::THREADS, YCfg<Rad<8, 10, 1>>::SMEM_BYTES, launch_y_80_1},
    {80, 2, 16, 5, 1, YCfg<Rad<16, 5, 1>>::THREADS, YCfg<Rad<16, 5, 1>>::SMEM_BYTES, launch_y_80_2},
    {81, 0, 9, 9, 1, YCfg<Rad<9, 9, 1>>::THREADS, YCfg<Rad<9, 9, 1>>::SMEM_BYTES, launch_y_81_0},
    {81, 1, 3, 3, 9, YCfg<Rad<3, 3, 9>>::THREADS, YCfg<Rad<3, 3, 9>>::SMEM_BYTES, launch_y_81_1},
    {84, 0, 12, 7, 1, YCfg<Rad<12, 7, 1>>::THREADS, YCfg<Rad<12, 7, 1>>::SMEM_BYTES, launch_y_84_0},
    {84, 1, 7, 12, 1, YCfg<Rad<7, 12, 1>>::THREADS, YCfg<Rad<7, 12, 1>>::SMEM_BYTES, launch_y_84_1},
    {84, 2, 14, 6, 1, YCfg<Rad<14, 6, 1>>::THREADS, YCfg<Rad<14, 6, 1>>::SMEM_BYTES, launch_y_84_2},
    {90, 0, 10, 9, 1, YCfg<Rad<10, 9, 1>>::THREADS, YCfg<Rad<10, 9, 1>>::SMEM_BYTES, launch_y_90_0},
    {90, 1, 9, 10, 1, YCfg<Rad<9, 10, 1>>::THREADS, YCfg<Rad<9, 10, 1>>::SMEM_BYTES, launch_y_90_1},
    {90, 2, 15, 6, 1, YCfg<Rad<15, 6, 1>>::THREADS, YCfg<Rad<15, 6, 1>>::SMEM_BYTES, launch_y_90_2},
    {96, 0, 12, 8, 1, YCfg<Rad<12, 8, 1>>::THREADS, YCfg<Rad<12, 8, 1>>::SMEM_BYTES, launch_y_96_0},
    {96, 1, 8, 12, 1, YCfg<Rad<8, 12, 1>>::THREADS, YCfg<Rad<8, 12, 1>>::SMEM_BYTES, launch_y_96_1},
    {96, 2, 16, 6, 1, YCfg<Rad<16, 6, 1>>::THREADS, YCfg<Rad<16, 6, 1>>::SMEM_BYTES, launch_y_96_2},
    {98, 0, 14, 7, 1, YCfg<Rad<14, 7, 1>>::THREADS, YCfg<Rad<14, 7, 1>>::SMEM_BYTES, launch_y_98_0},
    {98, 1, 7, 14, 1, YCfg<Rad<7, 14, 1>>::THREADS, YCfg<Rad<7, 14, 1>>::SMEM_BYTES, launch_y_98_1},
    {98, 2, 2, 7, 7, YCfg<Rad<2, 7, 7>>::THREADS, YCfg<Rad<2, 7, 7>>::SMEM_BYTES, launch_y_98_2},
    {100, 0, 10, 10, 1, YCfg<Rad<10, 10, 1>>::THREADS, YCfg<Rad<10, 10, 1>>::SMEM_BYTES, launch_y_100_0},
    {100, 1, 5, 4, 5, YCfg<Rad<5, 4, 5>>::THREADS, YCfg<Rad<5, 4, 5>>::SMEM_BYTES, launch_y_100_1},
    {100, 2, 4, 5, 5, YCfg<Rad<4, 5, 5>>::THREADS, YCfg<Rad<4, 5, 5>>::SMEM_BYTES, launch_y_100_2},
    {105, 0, 15, 7, 1, YCfg<Rad<15, 7, 1>>::THREADS, YCfg<Rad<15, 7, 1>>::SMEM_BYTES, launch_y_105_0},
    {105, 1, 7, 15, 1, YCfg<Rad<7, 15, 1>>::THREADS, YCfg<Rad<7, 15, 1>>::SMEM_BYTES, launch_y_105_1},
    {105, 2, 5, 3, 7, YCfg<Rad<5, 3, 7>>::THREADS, YCfg<Rad<5, 3, 7>>::SMEM_BYTES, launch_y_105_2},
    {108, 0, 12, 9, 1, YCfg<Rad<12, 9, 1>>::THREADS, YCfg<Rad<12, 9, 1>>::SMEM_BYTES, launch_y_108_0},
    {108, 1, 9, 12, 1, YCfg<Rad<9, 12, 1>>::THREADS, YCfg<Rad<9, 12, 1>>::SMEM_BYTES, launch_y_108_1},
    {108, 2, 6, 3, 6, YCfg<Rad<6, 3, 6>>::THREADS, YCfg<Rad<6, 3, 6>>::SMEM_BYTES, launch_y_108_2},
    {112, 0, 14, 8, 1, YCfg<Rad<14, 8, 1>>::THREADS, YCfg<Rad<14, 8, 1>>::SMEM_BYTES, launch_y_112_0},
    {112, 1, 8, 14, 1, YCfg<Rad<8, 14, 1>>::THREADS, YCfg<Rad<8, 14, 1>>::SMEM_BYTES, launch_y_112_1},
    {112, 2, 16, 7, 1, YCfg<Rad<16, 7, 1>>::THREADS, YCfg<Rad<16, 7, 1>>::SMEM_BYTES, launch_y_112_2},
    {120, 0, 12, 10, 1, YCfg<Rad<12, 10, 1>>::THREADS, YCfg<Rad<12, 10, 1>>::SMEM_BYTES, launch_y_120_0},
    {120, 1, 10, 12, 1, YCfg<Rad<10, 12, 1>>::THREADS, YCfg<Rad<10, 12, 1>>::SMEM_BYTES, launch_y_120_1},
    {120, 2, 15, 8, 1, YCfg<Rad<15, 8, 1>>::THREADS, YCfg<Rad<15, 8, 1>>::SMEM_BYTES, launch_y_120_2},
    {125, 0, 5, 5, 5, YCfg<Rad<5, 5, 5>>::THREADS, YCfg<Rad<5, 5, 5>>::SMEM_BYTES, launch_y_125_0},
    {126, 0, 14, 9, 1, YCfg<Rad<14, 9, 1>>::THREADS, YCfg<Rad<14, 9, 1>>::SMEM_BYTES, launch_y_126_0},
    {126, 1, 9, 14, 1, YCfg<Rad<9, 14, 1>>::THREADS, YCfg<Rad<9, 14, 1>>::SMEM_BYTES, launch_y_126_1},
    {126, 2, 7, 3, 6, YCfg<Rad<7, 3, 6>>::THREADS, YCfg<Rad<7, 3, 6>>::SMEM_BYTES, launch_y_126_2},
    {128, 0, 16, 8, 1, YCfg<Rad<16, 8, 1>>::THREADS, YCfg<Rad<16, 8, 1>>::SMEM_BYTES, launch_y_128_0},
    {128, 1, 8, 16, 1, YCfg<Rad<8, 16, 1>>::THREADS, YCfg<Rad<8, 16, 1>>::SMEM_BYTES, launch_y_128_1},
    {128, 2, 4, 4, 8, YCfg<Rad<4, 4, 8>>::THREADS, YCfg<Rad<4, 4, 8>>::SMEM_BYTES, launch_y_128_2},
    {135, 0, 15, 9, 1, YCfg<Rad<15, 9, 1>>::THREADS, YCfg<Rad<15, 9, 1>>::SMEM_BYTES, launch_y_135_0},
    {135, 1, 9, 15, 1, YCfg<Rad<9, 15, 1>>::THREADS, YCfg<Rad<9, 15, 1>>::SMEM_BYTES, launch_y_135_1},
    {135, 2, 5, 3, 9, YCfg<Rad<5, 3, 9>>::THREADS, YCfg<Rad<5, 3, 9>>::SMEM_BYTES, launch_y_135_2},
    {140, 0, 14, 10, 1, YCfg<Rad<14, 10, 1>>::THREADS, YCfg<Rad<14, 10, 1>>::SMEM_BYTES, launch_y_140_0},
    {140, 1, 10, 14, 1, YCfg<Rad<10, 14, 1>>::THREADS, YCfg<Rad<10, 14, 1>>::SMEM_BYTES, launch_y_140_1},
    {140, 2, 7, 4, 5, YCfg<Rad<7, 4, 5>>::THREADS, YCfg<Rad<7, 4, 5>>::SMEM_BYTES, launch_y_140_2},
    {144, 0, 12, 12, 1, YCfg<Rad<12, 12, 1>>::THREADS, YCfg<Rad<12, 12, 1>>::SMEM_BYTES, launch_y_144_0},
    {144, 1, 16, 9, 1, YCfg<Rad<16, 9, 1>>::THREADS, YCfg<Rad<16, 9, 1>>::SMEM_BYTES, launch_y_144_1},
    {144, 2, 9, 16, 1, YCfg<Rad<9, 16, 1>>::THREADS, YCfg<Rad<9, 16, 1>>::SMEM_BYTES, launch_y_144_2},
    {147, 0, 7, 3, 7, YCfg<Rad<7, 3, 7>>::THREADS, YCfg<Rad<7, 3, 7>>::SMEM_BYTES, launch_y_147_0},
    {147, 1, 3, 7, 7, YCfg<Rad<3, 7, 7>>::THREADS, YCfg<Rad<3, 7, 7>>::SMEM_BYTES, launch_y_147_1},
    {150, 0, 15, 10, 1, YCfg<Rad<15, 10, 1>>::THREADS, YCfg<Rad<15, 10, 1>>::SMEM_BYTES, launch_y_150_0},
    {150, 1, 10, 15, 1, YCfg<Rad<10, 15, 1>>::THREADS, YCfg<Rad<10, 15, 1>>::SMEM_BYTES, launch_y_150_1},
    {150, 2, 6, 5, 5, YCfg<Rad<6, 5, 5>>::THREADS, YCfg<Rad<6, 5, 5>>::SMEM_BYTES, launch_y_150_2},
    {160, 0, 16, 10, 1, YCfg<Rad<16, 10, 1>>::THREADS, YCfg<Rad<16, 10, 1>>::SMEM_BYTES, launch_y_160_0},
    {160, 1, 10, 16, 1, YCfg<Rad<10, 16, 1>>::THREADS, YCfg<Rad<10, 16, 1>>::SMEM_BYTES, launch_y_160_1},
    {160, 2, 8, 4, 5, YCfg<Rad<8, 4, 5>>::THREADS, YCfg<Rad<8, 4, 5>>::SMEM_BYTES, launch_y_160_2},
    {162, 0, 9, 3, 6, YCfg<Rad<9, 3, 6>>::THREADS, YCfg<Rad<9, 3, 6>>::SMEM_BYTES, launch_y_162_0},
    {162, 1, 6, 3, 9, YCfg<Rad<6, 3, 9>>::THREADS, YCfg<Rad<6, 3, 9>>::SMEM_BYTES, launch_y_162_1},
    {162, 2, 3, 6, 9, YCfg<Rad<3, 6, 9>>::THREADS, YCfg<Rad<3, 6, 9>>::SMEM_BYTES, launch_y_162_2},
    {168, 0, 14, 12, 1, YCfg<Rad<14, 12, 1>>::THREADS, YCfg<Rad<14, 12, 1>>::SMEM_BYTES, launch_y_168_0},
    {168, 1, 12, 14, 1, YCfg<Rad<12, 14, 1>>::THREADS, YCfg<Rad<12, 14, 1>>::SMEM_BYTES, launch_y_168_1},
    {168, 2, 7, 4, 6, YCfg<Rad<7, 4, 6>>::THREADS, YCfg<Rad<7, 4, 6>>::SMEM_BYTES, launch_y_168_2},
    {175, 0, 7, 5, 5, YCfg<Rad<7, 5, 5>>::THREADS, YCfg<Rad<7, 5, 5>>::SMEM_BYTES, launch_y_175_0},
    {175, 1, 5, 5, 7, YCfg<Rad<5, 5, 7>>::THREADS, YCfg<Rad<5, 5, 7>>::SMEM_BYTES, launch_y_175_1},
    {180, 0, 15, 12, 1, YCfg<Rad<15, 12, 1>>::THREADS, YCfg<Rad<15, 12, 1>>::SMEM_BYTES, launch_y_180_0},
    {180, 1, 12, 15, 1, YCfg<Rad<12, 15, 1>>::THREADS, YCfg<Rad<12, 15, 1>>::SMEM_BYTES, launch_y_180_1},
    {180, 2, 6, 5, 6, YCfg<Rad<6, 5, 6>>::THREADS, YCfg<Rad<6, 5, 6>>::SMEM_BYTES, launch_y_180_2},
    {189, 0, 9, 3, 7, YCfg<Rad<9, 3, 7>>::THREADS, YCfg<Rad<9, 3, 7>>::SMEM_BYTES, launch_y_189_0},
    {189, 1, 7, 3, 9, YCfg<Rad<7, 3, 9>>::THREADS, YCfg<Rad<7, 3, 9>>::SMEM_BYTES, launch_y_189_1},
    {189, 2, 3, 7, 9, YCfg<Rad<3, 7, 9>>::THREADS, YCfg<Rad<3, 7, 9>>::SMEM_BYTES, launch_y_189_2},
    {192, 0, 16, 12, 1, YCfg<Rad<16, 12, 1>>::THREADS, YCfg<Rad<16, 12, 1>>::SMEM_BYTES, launch_y_192_0},
    {192, 1, 12, 16, 1, YCfg<Rad<12, 16, 1>>::THREADS, YCfg<Rad<12, 16, 1>>::SMEM_BYTES, launch_y_192_1},
    {192, 2, 8, 4, 6, YCfg<Rad<8, 4, 6>>::THREADS, YCfg<Rad<8, 4, 6>>::SMEM_BYTES, launch_y_192_2},
    {196, 0, 14, 14, 1, YCfg<Rad<14, 14, 1>>::THREADS, YCfg<Rad<14, 14, 1>>::SMEM_BYTES, launch_y_196_0},
    {196, 1, 7, 4, 7, YCfg<Rad<7, 4, 7>>::THREADS, YCfg<Rad<7, 4, 7>>::SMEM_BYTES, launch_y_196_1},
    {196, 2, 4, 7, 7, YCfg<Rad<4, 7, 7>>::THREADS, YCfg<Rad<4, 7, 7>>::SMEM_BYTES, launch_y_196_2},
    {200, 0, 8, 5, 5, YCfg<Rad<8, 5, 5>>::THREADS, YCfg<Rad<8, 5, 5>>::SMEM_BYTES, launch_y_200_0},
    {200, 1, 5, 5, 8, YCfg<Rad<5, 5, 8>>::THREADS, YCfg<Rad<5, 5, 8>>::SMEM_BYTES, launch_y_200_1},
    {200, 2, 10, 4, 5, YCfg<Rad<10, 4, 5>>::THREADS, YCfg<Rad<10, 4, 5>>::SMEM_BYTES, launch_y_200_2},
    {210, 0, 15, 14, 1, YCfg<Rad<15, 14, 1>>::THREADS, YCfg<Rad<15, 14, 1>>::SMEM_BYTES, launch_y_210_0},
    {210, 1, 14, 15, 1, YCfg<Rad<14, 15, 1>>::THREADS, YCfg<Rad<14, 15, 1>>::SMEM_BYTES, launch_y_210_1},
    {210, 2, 7, 5, 6, YCfg<Rad<7, 5, 6>>::THREADS, YCfg<Rad<7, 5, 6>>::SMEM_BYTES, launch_y_210_2},
    {216, 0, 6, 6, 6, YCfg<Rad<6, 6, 6>>::THREADS, YCfg<Rad<6, 6, 6>>::SMEM_BYTES, launch_y_216_0},
    {216, 1, 9, 4, 6, YCfg<Rad<9, 4, 6>>::THREADS, YCfg<Rad<9, 4, 6>>::SMEM_BYTES, launch_y_216_1},
    {216, 2, 4, 6, 9, YCfg<Rad<4, 6, 9>>::THREADS, YCfg<Rad<4, 6, 9>>::SMEM_BYTES, launch_y_216_2},
    {224, 0, 16, 14, 1, YCfg<Rad<16, 14, 1>>::THREADS, YCfg<Rad<16, 14, 1>>::SMEM_BYTES, launch_y_224_0},
    {224, 1, 14, 16, 1, YCfg<Rad<14, 16, 1>>::THREADS, YCfg<Rad<14, 16, 1>>::SMEM_BYTES, launch_y_224_1},
    {224, 2, 8, 4, 7, YCfg<Rad<8, 4, 7>>::THREADS, YCfg<Rad<8, 4, 7>>::SMEM_BYTES, launch_y_224_2},
    {225, 0, 15, 15, 1, YCfg<Rad<15, 15, 1>>::THREADS, YCfg<Rad<15, 15, 1>>::SMEM_BYTES, launch_y_225_0},
    {225, 1, 9, 5, 5, YCfg<Rad<9, 5, 5>>::THREADS, YCfg<Rad<9, 5, 5>>::SMEM_BYTES, launch_y_225_1},
    {225, 2, 5, 5, 9, YCfg<Rad<5, 5, 9>>::THREADS, YCfg<Rad<5, 5, 9>>::SMEM_BYTES, launch_y_225_2},
    {240, 0, 16, 15, 1, YCfg<Rad<16, 15, 1>>::THREADS, YCfg<Rad<16, 15, 1>>::SMEM_BYTES, launch_y_240_0},
    {240, 1, 15, 16, 1, YCfg<Rad<15, 16, 1>>::THREADS, YCfg<Rad<15, 16, 1>>::SMEM_BYTES, launch_y_240_1},
    {240, 2, 8, 5, 6, YCfg<Rad<8, 5, 6>>::THREADS, YCfg<Rad<8, 5, 6>>::SMEM_BYTES, launch_y_240_2},
    {243, 0, 9, 3, 9, YCfg<Rad<9, 3, 9>>::THREADS, YCfg<Rad<9, 3, 9>>::SMEM_BYTES, launch_y_243_0},
    {243, 1, 3, 9, 9, YCfg<Rad<3, 9, 9>>::THREADS, YCfg<Rad<3, 9, 9>>::SMEM_BYTES, launch_y_243_1},
    {245, 0, 7, 5, 7, YCfg<Rad<7, 5, 7>>::THREADS, YCfg<Rad<7, 5, 7>>::SMEM_BYTES, launch_y_245_0},
    {245, 1, 5, 7, 7, YCfg<Rad<5, 7, 7>>::THREADS, YCfg<Rad<5, 7, 7>>::SMEM_BYTES, launch_y_245_1},
    {250, 0, 10, 5, 5, YCfg<Rad<10, 5, 5>>::THREADS, YCfg<Rad<10, 5, 5>>::SMEM_BYTES, launch_y_250_0},
    {250, 1, 5, 5, 10, YCfg<Rad<5, 5, 10>>::THREADS, YCfg<Rad<5, 5, 10>>::SMEM_BYTES, launch_y_250_1},
    {252, 0, 7, 6, 6, YCfg<Rad<7, 6, 6>>::THREADS, YCfg<Rad<7, 6, 6>>::SMEM_BYTES, launch_y_252_0},
    {252, 1, 6, 6, 7, YCfg<Rad<6, 6, 7>>::THREADS, YCfg<Rad<6, 6, 7>>::SMEM_BYTES, launch_y_252_1},
    {252, 2, 9, 4, 7, YCfg<Rad<9, 4, 7>>::THREADS, YCfg<Rad<9, 4, 7>>::SMEM_BYTES, launch_y_252_2},
    {256, 0, 16, 16, 1, YCfg<Rad<16, 16, 1>>::THREADS, YCfg<Rad<16, 16, 1>>::SMEM_BYTES, launch_y_256_0},
    {256, 1, 8, 4, 8, YCfg<Rad<8, 4, 8>>::THREADS, YCfg<Rad<8, 4, 8>>::SMEM_BYTES, launch_y_256_1},
    {256, 2, 4, 8, 8, YCfg<Rad<4, 8, 8>>::THREADS, YCfg<Rad<4, 8, 8>>::SMEM_BYTES, launch_y_256_2},
    {270, 0, 9, 5, 6, YCfg<Rad<9, 5, 6>>::THREADS, YCfg<Rad<9, 5, 6>>::SMEM_BYTES, launch_y_270_0},
    {270, 1, 6, 5, 9, YCfg<Rad<6, 5, 9>>::THREADS, YCfg<Rad<6, 5, 9>>::SMEM_BYTES, launch_y_270_1},
    {270, 2, 5, 6, 9, YCfg<Rad<5, 6, 9>>::THREADS, YCfg<Rad<5, 6, 9>>::SMEM_BYTES, launch_y_270_2},
    {280, 0, 8, 5, 7, YCfg<Rad<8, 5, 7>>::THREADS, YCfg<Rad<8, 5, 7>>::SMEM_BYTES, launch_y_280_0},
    {280, 1, 7, 5, 8, YCfg<Rad<7, 5, 8>>::THREADS, YCfg<Rad<7, 5, 8>>::SMEM_BYTES, launch_y_280_1},
    {280, 2, 5, 7, 8, YCfg<Rad<5, 7, 8>>::THREADS, YCfg<Rad<5, 7, 8>>::SMEM_BYTES, launch_y_280_2},
    {288, 0, 8, 6, 6, YCfg<Rad<8, 6, 6>>::THREADS, YCfg<Rad<8, 6, 6>>::SMEM_BYTES, launch_y_288_0},
    {288, 1, 6, 6, 8, YCfg<Rad<6, 6, 8>>::THREADS, YCfg<Rad<6, 6, 8>>::SMEM_BYTES, launch_y_288_1},
    {288, 2, 9, 4, 8, YCfg<Rad<9, 4, 8>>::THREADS, YCfg<Rad<9, 4, 8>>::SMEM_BYTES, launch_y_288_2},
    {294, 0, 7, 6, 7, YCfg<Rad<7, 6, 7>>::THREADS, YCfg<Rad<7, 6, 7>>::SMEM_BYTES, launch_y_294_0},
    {294, 1, 6, 7, 7, YCfg<Rad<6, 7, 7>>::THREADS, YCfg<Rad<6, 7, 7>>::SMEM_BYTES, launch_y_294_1},
    {294, 2, 14, 3, 7, YCfg<Rad<14, 3, 7>>::THREADS, YCfg<Rad<14, 3, 7>>::SMEM_BYTES, launch_y_294_2},
    {300, 0, 10, 5, 6, YCfg<Rad<10, 5, 6>>::THREADS, YCfg<Rad<10, 5, 6>>::SMEM_BYTES, launch_y_300_0},
    {300, 1, 6, 5, 10, YCfg<Rad<6, 5, 10>>::THREADS, YCfg<Rad<6, 5, 10>>::SMEM_BYTES, launch_y_300_1},
    {300, 2, 5, 6, 10, YCfg<Rad<5, 6, 10>>::THREADS, YCfg<Rad<5, 6, 10>>::SMEM_BYTES, launch_y_300_2},
    {315, 0, 9, 5, 7, YCfg<Rad<9, 5, 7>>::THREADS, YCfg<Rad<9, 5, 7>>::SMEM_BYTES, launch_y_315_0},
    {315, 1, 7, 5, 9, YCfg<Rad<7, 5, 9>>::THREADS, YCfg<Rad<7, 5, 9>>::SMEM_BYTES, launch_y_315_1},
    {315, 2, 5, 7, 9, YCfg<Rad<5, 7, 9>>::THREADS, YCfg<Rad<5, 7, 9>>::SMEM_BYTES, launch_y_315_2},
    {320, 0, 8, 5, 8, YCfg<Rad<8, 5, 8>>::THREADS, YCfg<Rad<8, 5, 8>>::SMEM_BYTES, launch_y_320_0},
    {320, 1, 5, 8, 8, YCfg<Rad<5, 8, 8>>::THREADS, YCfg<Rad<5, 8, 8>>::SMEM_BYTES, launch_y_320_1},
    {320, 2, 10, 4, 8, YCfg<Rad<10, 4, 8>>::THREADS, YCfg<Rad<10, 4, 8>>::SMEM_BYTES, launch_y_320_2},
    {324, 0, 9, 6, 6, YCfg<Rad<9, 6, 6>>::THREADS, YCfg<Rad<9, 6, 6>>::SMEM_BYTES, launch_y_324_0},
    {324, 1, 6, 6, 9, YCfg<Rad<6, 6, 9>>::THREADS, YCfg<Rad<6, 6, 9>>::SMEM_BYTES, launch_y_324_1},
    {324, 2, 4, 9, 9, YCfg<Rad<4, 9, 9>>::THREADS, YCfg<Rad<4, 9, 9>>::SMEM_BYTES, launch_y_324_2},
    {336, 0, 8, 6, 7, YCfg<Rad<8, 6, 7>>::THREADS, YCfg<Rad<8, 6, 7>>::SMEM_BYTES, launch_y_336_0},
    {336, 1, 7, 6, 8, YCfg<Rad<7, 6, 8>>::THREADS, YCfg<Rad<7, 6, 8>>::SMEM_BYTES, launch_y_336_1},
    {336, 2, 6, 7, 8, YCfg<Rad<6, 7, 8>>::THREADS, YCfg<Rad<6, 7, 8>>::SMEM_BYTES, launch_y_336_2},
    {343, 0, 7, 7, 7, YCfg<Rad<7, 7, 7>>::THREADS, YCfg<Rad<7, 7, 7>>::SMEM_BYTES, launch_y_343_0},
    {350, 0, 10, 5, 7, YCfg<Rad<10, 5, 7>>::THREADS, YCfg<Rad<10, 5, 7>>::SMEM_BYTES, launch_y_350_0},
    {350, 1, 7, 5, 10, YCfg<Rad<7, 5, 10>>::THREADS, YCfg<Rad<7, 5, 10>>::SMEM_BYTES, launch_y_350_1},
    {350, 2, 5, 7, 10, YCfg<Rad<5, 7, 10>>::THREADS, YCfg<Rad<5, 7, 10>>::SMEM_BYTES, launch_y_350_2},
    {360, 0, 10, 6, 6, YCfg<Rad<10, 6, 6>>::THREADS, YCfg<Rad<10, 6, 6>>::SMEM_BYTES, launch_y_360_0},
    {360, 1, 6, 6, 10, YCfg<Rad<6, 6, 10>>::THREADS, YCfg<Rad<6, 6, 10>>::SMEM_BYTES, launch_y_360_1},
    {360, 2, 9, 5, 8, YCfg<Rad<9, 5, 8>>::THREADS, YCfg<Rad<9, 5, 8>>::SMEM_BYTES, launch_y_360_2},
    {375, 0, 15, 5, 5, YCfg<Rad<15, 5, 5>>::THREADS, YCfg<Rad<15, 5, 5>>::SMEM_BYTES, launch_y_375_0},
    {375, 1, 5, 5, 15, YCfg<Rad<5, 5, 15>>::THREADS, YCfg<Rad<5, 5, 15>>::SMEM_BYTES, launch_y_375_1},
    {378, 0, 9, 6, 7, YCfg<Rad<9, 6, 7>>::THREADS, YCfg<Rad<9, 6, 7>>::SMEM_BYTES, launch_y_378_0},
    {378, 1, 7, 6, 9, YCfg<Rad<7, 6, 9>>::THREADS, YCfg<Rad<7, 6, 9>>::SMEM_BYTES, launch_y_378_1},
    {378, 2, 6, 7, 9, YCfg<Rad<6, 7, 9>>::THREADS, YCfg<Rad<6, 7, 9>>::SMEM_BYTES, launch_y_378_2},
    {384, 0, 8, 6, 8, YCfg<Rad<8, 6, 8>>::THREADS, YCfg<Rad<8, 6, 8>>::SMEM_BYTES, launch_y_384_0},
    {384, 1, 6, 8, 8, YCfg<Rad<6, 8, 8>>::THREADS, YCfg<Rad<6, 8, 8>>::SMEM_BYTES, launch_y_384_1},
    {384, 2, 12, 4, 8, YCfg<Rad<12, 4, 8>>::THREADS, YCfg<Rad<12, 4, 8>>::SMEM_BYTES, launch_y_384_2},
    {392, 0, 8, 7, 7, YCfg<Rad<8, 7, 7>>::THREADS, YCfg<Rad<8, 7, 7>>::SMEM_BYTES, launch_y_392_0},
    {392, 1, 7, 7, 8, YCfg<Rad<7, 7, 8>>::THREADS, YCfg<Rad<7, 7, 8>>::SMEM_BYTES, launch_y_392_1},
    {392, 2, 14, 4, 7, YCfg<Rad<14, 4, 7>>::THREADS, YCfg<Rad<14, 4, 7>>::SMEM_BYTES, launch_y_392_2},
    {400, 0, 10, 5, 8, YCfg<Rad<10, 5, 8>>::THREADS, YCfg<Rad<10, 5, 8>>::SMEM_BYTES, launch_y_400_0},
    {400, 1, 8, 5, 10, YCfg<Rad<8, 5, 10>>::THREADS, YCfg<Rad<8, 5, 10>>::SMEM_BYTES, launch_y_400_1},
    {400, 2, 5, 8, 10, YCfg<Rad<5, 8, 10>>::THREADS, YCfg<Rad<5, 8, 10>>::SMEM_BYTES, launch_y_400_2},
    {405, 0, 9, 5, 9, YCfg<Rad<9, 5, 9>>::THREADS, YCfg<Rad<9, 5, 9>>::SMEM_BYTES, launch_y_405_0},
    {405, 1, 5, 9, 9, YCfg<Rad<5, 9, 9>>::THREADS, YCfg<Rad<5, 9, 9>>::SMEM_BYTES, launch_y_405_1},
    {405, 2, 15, 3, 9, YCfg<Rad<15, 3, 9>>::THREADS, YCfg<Rad<15, 3, 9>>::SMEM_BYTES, launch_y_405_2},
    {420, 0, 10, 6, 7, YCfg<Rad<10, 6, 7>>::THREADS, YCfg<Rad<10, 6, 7>>::SMEM_BYTES, launch_y_420_0},
    {420, 1, 7, 6, 10, YCfg<Rad<7, 6, 10>>::THREADS, YCfg<Rad<7, 6, 10>>::SMEM_BYTES, launch_y_420_1},
    {420, 2, 6, 7, 10, YCfg<Rad<6, 7, 10>>::THREADS, YCfg<Rad<6, 7, 10>>::SMEM_BYTES, launch_y_420_2},
    {432, 0, 9, 6, 8, YCfg<Rad<9, 6, 8>>::THREADS, YCfg<Rad<9, 6, 8>>::SMEM_BYTES, launch_y_432_0},
    {432, 1, 8, 6, 9, YCfg<Rad<8, 6, 9>>::THREADS, YCfg<Rad<8, 6, 9>>::SMEM_BYTES, launch_y_432_1},
    {432, 2, 6, 8, 9, YCfg<Rad<6, 8, 9>>::THREADS, YCfg<Rad<6, 8, 9>>::SMEM_BYTES, launch_y_432_2},
    {441, 0, 9, 7, 7, YCfg<Rad<9, 7, 7>>::THREADS, YCfg<Rad<9, 7, 7>>::SMEM_BYTES, launch_y_441_0},
    {441, 1, 7, 7, 9, YCfg<Rad<7, 7, 9>>::THREADS, YCfg<Rad<7, 7, 9>>::SMEM_BYTES, launch_y_441_1},
    {448, 0, 8, 7, 8, YCfg<Rad<8, 7, 8>>::THREADS, YCfg<Rad<8, 7, 8>>::SMEM_BYTES, launch_y_448_0},
    {448, 1, 7, 8, 8, YCfg<Rad<7, 8, 8>>::THREADS, YCfg<Rad<7, 8, 8>>::SMEM_BYTES, launch_y_448_1},
    {448, 2, 14, 4, 8, YCfg<Rad<14, 4, 8>>::THREADS, YCfg<Rad<14, 4, 8>>::SMEM_BYTES, launch_y_448_2},
    {450, 0, 10, 5, 9, YCfg<Rad<10, 5, 9>>::THREADS, YCfg<Rad<10, 5, 9>>::SMEM_BYTES, launch_y_450_0},
    {450, 1, 9, 5, 10, YCfg<Rad<9, 5, 10>>::THREADS, YCfg<Rad<9, 5, 10>>::SMEM_BYTES, launch_y_450_1},
    {450, 2, 5, 9, 10, YCfg<Rad<5, 9, 10>>::THREADS, YCfg<Rad<5, 9, 10>>::SMEM_BYTES, launch_y_450_2},
    {480, 0, 10, 6, 8, YCfg<Rad<10, 6, 8>>::THREADS, YCfg<Rad<10, 6, 8>>::SMEM_BYTES, launch_y_480_0},
    {480, 1, 8, 6, 10, YCfg<Rad<8, 6, 10>>::THREADS, YCfg<Rad<8, 6, 10>>::SMEM_BYTES, launch_y_480_1},
    {480, 2, 6, 8, 10, YCfg<Rad<6, 8, 10>>::THREADS, YCfg<Rad<6, 8, 10>>::SMEM_BYTES, launch_y_480_2},
    {486, 0, 9, 6, 9, YCfg<Rad<9, 6, 9>>::THREADS, YCfg<Rad<9, 6, 9>>::SMEM_BYTES, launch_y_486_0},
    {486, 1, 6, 9, 9, YCfg<Rad<6, 9, 9>>::THREADS, YCfg<Rad<6, 9, 9>>::SMEM_BYTES, launch_y_486_1},
    {490, 0, 10, 7, 7, YCfg<Rad<10, 7, 7>>::THREADS, YCfg<Rad<10, 7, 7>>::SMEM_BYTES, launch_y_490_0},
    {490, 1, 7, 7, 10, YCfg<Rad<7, 7, 10>>::THREADS, YCfg<Rad<7, 7, 10>>::SMEM_BYTES, launch_y_490_1},
    {490, 2, 14, 5, 7, YCfg<Rad<14, 5, 7>>::THREADS, YCfg<Rad<14, 5, 7>>::SMEM_BYTES, launch_y_490_2},
    {500, 0, 10, 5, 10, YCfg<Rad<10, 5, 10>>::THREADS, YCfg<Rad<10, 5, 10>>::SMEM_BYTES, launch_y_500_0},
    {500, 1, 5, 10, 10, YCfg<Rad<5, 10, 10>>::THREADS, YCfg<Rad<5, 10, 10>>::SMEM_BYTES, launch_y_500_1},
    {504, 0, 9, 7, 8, YCfg<Rad<9, 7, 8>>::THREADS, YCfg<Rad<9, 7, 8>>::SMEM_BYTES, launch_y_504_0},
    {504, 1, 8, 7, 9, YCfg<Rad<8, 7, 9>>::THREADS, YCfg<Rad<8, 7, 9>>::SMEM_BYTES, launch_y_504_1},
    {504, 2, 7, 8, 9, YCfg<Rad<7, 8, 9>>::THREADS, YCfg<Rad<7, 8, 9>>::SMEM_BYTES, launch_y_504_2},
    {512, 0, 8, 8, 8, YCfg<Rad<8, 8, 8>>::THREADS, YCfg<Rad<8, 8, 8>>::SMEM_BYTES, launch_y_512_0},
    {512, 1, 16, 4, 8, YCfg<Rad<16, 4, 8>>::THREADS, YCfg<Rad<16, 4, 8>>::SMEM_BYTES, launch_y_512_1},
    {512, 2, 4, 8, 16, YCfg<Rad<4, 8, 16>>::THREADS, YCfg<Rad<4, 8, 16>>::SMEM_BYTES, launch_y_512_2},
    {525, 0, 15, 5, 7, YCfg<Rad<15, 5, 7>>::THREADS, YCfg<Rad<15, 5, 7>>::SMEM_BYTES, launch_y_525_0},
    {525, 1, 7, 5, 15, YCfg<Rad<7, 5, 15>>::THREADS, YCfg<Rad<7, 5, 15>>::SMEM_BYTES, launch_y_525_1},
    {525, 2, 5, 7, 15, YCfg<Rad<5, 7, 15>>::THREADS, YCfg<Rad<5, 7, 15>>::SMEM_BYTES, launch_y_525_2},
    {540, 0, 10, 6, 9, YCfg<Rad<10, 6, 9>>::THREADS, YCfg<Rad<10, 6, 9>>::SMEM_BYTES, launch_y_540_0},
    {540, 1, 9, 6, 10, YCfg<Rad<9, 6, 10>>::THREADS, YCfg<Rad<9, 6, 10>>::SMEM_BYTES, launch_y_540_1},
    {540, 2, 6, 9, 10, YCfg<Rad<6, 9, 10>>::THREADS, YCfg<Rad<6, 9, 10>>::SMEM_BYTES, launch_y_540_2},
    {560, 0, 10, 7, 8, YCfg<Rad<10, 7, 8>>::THREADS, YCfg<Rad<10, 7, 8>>::SMEM_BYTES, launch_y_560_0},
    {560, 1, 8, 7, 10, YCfg<Rad<8, 7, 10>>::THREADS, YCfg<Rad<8, 7, 10>>::SMEM_BYTES, launch_y_560_1},
    {560, 2, 7, 8, 10, YCfg<Rad<7, 8, 10>>::THREADS, YCfg<Rad<7, 8, 10>>::SMEM_BYTES, launch_y_560_2},
    {567, 0, 9, 7, 9, YCfg<Rad<9, 7, 9>>::THREADS, YCfg<Rad<9, 7, 9>>::SMEM_BYTES, launch_y_567_0},
    {567, 1, 7, 9, 9, YCfg<Rad<7, 9, 9>>::THREADS, YCfg<Rad<7, 9, 9>>::SMEM_BYTES, launch_y_567_1},
    {576, 0, 9, 8, 8, YCfg<Rad<9, 8, 8>>::THREADS, YCfg<Rad<9, 8, 8>>::SMEM_BYTES, launch_y_576_0},
    {576, 1, 8, 8, 9, YCfg<Rad<8, 8, 9>>::THREADS, YCfg<Rad<8, 8, 9>>::SMEM_BYTES, launch_y_576_1},
    {576, 2, 12, 6, 8, YCfg<Rad<12, 6, 8>>::THREADS, YCfg<Rad<12, 6, 8>>::SMEM_BYTES, launch_y_576_2},
    {588, 0, 12, 7, 7, YCfg<Rad<12, 7, 7>>::THREADS, YCfg<Rad<12, 7, 7>>::SMEM_BYTES, launch_y_588_0},
    {588, 1, 7, 7, 12, YCfg<Rad<7, 7, 12>>::THREADS, YCfg<Rad<7, 7, 12>>::SMEM_BYTES, launch_y_588_1},
    {588, 2, 14, 6, 7, YCfg<Rad<14, 6, 7>>::THREADS, YCfg<Rad<14, 6, 7>>::SMEM_BYTES, launch_y_588_2},
    {600, 0, 10, 6, 10, YCfg<Rad<10, 6, 10>>::THREADS, YCfg<Rad<10, 6, 10>>::SMEM_BYTES, launch_y_600_0},
    {600, 1, 6, 10, 10, YCfg<Rad<6, 10, 10>>::THREADS, YCfg<Rad<6, 10, 10>>::SMEM_BYTES, launch_y_600_1},
    {600, 2, 12, 5, 10, YCfg<Rad<12, 5, 10>>::THREADS, YCfg<Rad<12, 5, 10>>::SMEM_BYTES, launch_y_600_2},
    {630, 0, 10, 7, 9, YCfg<Rad<10, 7, 9>>::THREADS, YCfg<Rad<10, 7, 9>>::SMEM_BYTES, launch_y_630_0},
    {630, 1, 9, 7, 10, YCfg<Rad<9, 7, 10>>::THREADS, YCfg<Rad<9, 7, 10>>::SMEM_BYTES, launch_y_630_1},
    {630, 2, 7, 9, 10, YCfg<Rad<7, 9, 10>>::THREADS, YCfg<Rad<7, 9, 10>>::SMEM_BYTES, launch_y_630_2},
    {640, 0, 10, 8, 8, YCfg<Rad<10, 8, 8>>::THREADS, YCfg<Rad<10, 8, 8>>::SMEM_BYTES, launch_y_640_0},
    {640, 1, 8, 8, 10, YCfg<Rad<8, 8, 10>>::THREADS, YCfg<Rad<8, 8, 10>>::SMEM_BYTES, launch_y_640_1},
    {640, 2, 16, 5, 8, YCfg<Rad<16, 5, 8>>::THREADS, YCfg<Rad<16, 5, 8>>::SMEM_BYTES, launch_y_640_2},
    {648, 0, 9, 8, 9, YCfg<Rad<9, 8, 9>>::THREADS, YCfg<Rad<9, 8, 9>>::SMEM_BYTES, launch_y_648_0},
    {648, 1, 8, 9, 9, YCfg<Rad<8, 9, 9>>::THREADS, YCfg<Rad<8, 9, 9>>::SMEM_BYTES, launch_y_648_1},
    {648, 2, 12, 6, 9, YCfg<Rad<12, 6, 9>>::THREADS, YCfg<Rad<12, 6, 9>>::SMEM_BYTES, launch_y_648_2},
    {672, 0, 12, 7, 8, YCfg<Rad<12, 7, 8>>::THREADS, YCfg<Rad<12, 7, 8>>::SMEM_BYTES, launch_y_672_0},
    {672, 1, 8, 7, 12, YCfg<Rad<8, 7, 12>>::THREADS, YCfg<Rad<8, 7, 12>>::SMEM_BYTES, launch_y_672_1},
    {672, 2, 7, 8, 12, YCfg<Rad<7, 8, 12>>::THREADS, YCfg<Rad<7, 8, 12>>::SMEM_BYTES, launch_y_672_2},
    {675, 0, 15, 5, 9, YCfg<Rad<15, 5, 9>>::THREADS, YCfg<Rad<15, 5, 9>>::SMEM_BYTES, launch_y_675_0},
    {675, 1, 9, 5, 15, YCfg<Rad<9, 5, 15>>::THREADS, YCfg<Rad<9, 5, 15>>::SMEM_BYTES, launch_y_675_1},
    {675, 2, 5, 9, 15, YCfg<Rad<5, 9, 15>>::THREADS, YCfg<Rad<5, 9, 15>>::SMEM_BYTES, launch_y_675_2},
    {686, 0, 14, 7, 7, YCfg<Rad<14, 7, 7>>::THREADS, YCfg<Rad<14, 7, 7>>::SMEM_BYTES, launch_y_686_0},
    {686, 1, 7, 7, 14, YCfg<Rad<7, 7, 14>>::THREADS, YCfg<Rad<7, 7, 14>>::SMEM_BYTES, launch_y_686_1},
    {700, 0, 10, 7, 10, YCfg<Rad<10, 7, 10>>::THREADS, YCfg<Rad<10, 7, 10>>::SMEM_BYTES, launch_y_700_0},
    {700, 1, 7, 10, 10, YCfg<Rad<7, 10, 10>>::THREADS, YCfg<Rad<7, 10, 10>>::SMEM_BYTES, launch_y_700_1},
    {700, 2, 14, 5, 10, YCfg<Rad<14, 5, 10>>::THREADS, YCfg<Rad<14, 5, 10>>::SMEM_BYTES, launch_y_700_2},
    {720, 0, 10, 8, 9, YCfg<Rad<10, 8, 9>>::THREADS, YCfg<Rad<10, 8, 9>>::SMEM_BYTES, launch_y_720_0},
    {720, 1, 9, 8, 10, YCfg<Rad<9, 8, 10>>::THREADS, YCfg<Rad<9, 8, 10>>::SMEM_BYTES, launch_y_720_1},
    {720, 2, 8, 9, 10, YCfg<Rad<8, 9, 10>>::THREADS, YCfg<Rad<8, 9, 10>>::SMEM_BYTES, launch_y_720_2},
    {729, 0, 9, 9, 9, YCfg<Rad<9, 9, 9>>::THREADS, YCfg<Rad<9, 9, 9>>::SMEM_BYTES, launch_y_729_0},
    {735, 0, 15, 7, 7, YCfg<Rad<15, 7, 7>>::THREADS, YCfg<Rad<15, 7, 7>>::SMEM_BYTES, launch_y_735_0},
    {735, 1, 7, 7, 15, YCfg<Rad<7, 7, 15>>::THREADS, YCfg<Rad<7, 7, 15>>::SMEM_BYTES, launch_y_735_1},
    {750, 0, 15, 5, 10, YCfg<Rad<15, 5, 10>>::THREADS, YCfg<Rad<15, 5, 10>>::SMEM_BYTES, launch_y_750_0},
    {750, 1, 10, 5, 15, YCfg<Rad<10, 5, 15>>::THREADS, YCfg<Rad<10, 5, 15>>::SMEM_BYTES, launch_y_750_1},
    {750, 2, 5, 10, 15, YCfg<Rad<5, 10, 15>>::THREADS, YCfg<Rad<5, 10, 15>>::SMEM_BYTES, launch_y_750_2},
    {756, 0, 12, 7, 9, YCfg<Rad<12, 7, 9>>::THREADS, YCfg<Rad<12, 7, 9>>::SMEM_BYTES, launch_y_756_0},
    {756, 1, 9, 7, 12, YCfg<Rad<9, 7, 12>>::THREADS, YCfg<Rad<9, 7, 12>>::SMEM_BYTES, launch_y_756_1},
    {756, 2, 7, 9, 12, YCfg<Rad<7, 9, 12>>::THREADS, YCfg<Rad<7, 9, 12>>::SMEM_BYTES, launch_y_756_2},
    {768, 0, 12, 8, 8, YCfg<Rad<12, 8, 8>>::THREADS, YCfg<Rad<12, 8, 8>>::SMEM_BYTES, launch_y_768_0},
    {768, 1, 8, 8, 12, YCfg<Rad<8, 8, 12>>::THREADS, YCfg<Rad<8, 8, 12>>::SMEM_BYTES, launch_y_768_1},
    {768, 2, 16, 6, 8, YCfg<Rad<16, 6, 8>>::THREADS, YCfg<Rad<16, 6, 8>>::SMEM_BYTES, launch_y_768_2},
    {784, 0, 14, 7, 8, YCfg<Rad<14, 7, 8>>::THREADS, YCfg<Rad<14, 7, 8>>::SMEM_BYTES, launch_y_784_0},
    {784, 1, 8, 7, 14, YCfg<Rad<8, 7, 14>>::THREADS, YCfg<Rad<8, 7, 14>>::SMEM_BYTES, launch_y_784_1},
    {784, 2, 7, 8, 14, YCfg<Rad<7, 8, 14>>::THREADS, YCfg<Rad<7, 8, 14>>::SMEM_BYTES, launch_y_784_2},
    {800, 0, 10, 8, 10, YCfg<Rad<10, 8, 10>>::THREADS, YCfg<Rad<10, 8, 10>>::SMEM_BYTES, launch_y_800_0},
    {800, 1, 8, 10, 10, YCfg<Rad<8, 10, 10>>::THREADS, YCfg<Rad<8, 10, 10>>::SMEM_BYTES, launch_y_800_1},
    {800, 2, 16, 5, 10, YCfg<Rad<16, 5, 10>>::THREADS, YCfg<Rad<16, 5, 10>>::SMEM_BYTES, launch_y_800_2},
    {810, 0, 10, 9, 9, YCfg<Rad<10, 9, 9>>::THREADS, YCfg<Rad<10, 9, 9>>::SMEM_BYTES, launch_y_810_0},
    {810, 1, 9, 9, 10, YCfg<Rad<9, 9, 10>>::THREADS, YCfg<Rad<9, 9, 10>>::SMEM_BYTES, launch_y_810_1},
    {810, 2, 15, 6, 9, YCfg<Rad<15, 6, 9>>::THREADS, YCfg<Rad<15, 6, 9>>::SMEM_BYTES, launch_y_810_2},
    {840, 0, 12, 7, 10, YCfg<Rad<12, 7, 10>>::THREADS, YCfg<Rad<12, 7, 10>>::SMEM_BYTES, launch_y_840_0},
    {840, 1, 10, 7, 12, YCfg<Rad<10, 7, 12>>::THREADS, YCfg<Rad<10, 7, 12>>::SMEM_BYTES, launch_y_840_1},
    {840, 2, 7, 10, 12, YCfg<Rad<7, 10, 12>>::THREADS, YCfg<Rad<7, 10, 12>>::SMEM_BYTES, launch_y_840_2},
    {864, 0, 12, 8, 9, YCfg<Rad<12, 8, 9>>::THREADS, YCfg<Rad<12, 8, 9>>::SMEM_BYTES, launch_y_864_0},
    {864, 1, 9, 8, 12, YCfg<Rad<9, 8, 12>>::THREADS, YCfg<Rad<9, 8, 12>>::SMEM_BYTES, launch_y_864_1},
    {864, 2, 8, 9, 12, YCfg<Rad<8, 9, 12>>::THREADS, YCfg<Rad<8, 9, 12>>::SMEM_BYTES, launch_y_864_2},
    {882, 0, 14, 7, 9, YCfg<Rad<14, 7, 9>>::THREADS, YCfg<Rad<14, 7, 9>>::SMEM_BYTES, launch_y_882_0},
    {882, 1, 9, 7, 14, YCfg<Rad<9, 7, 14>>::THREADS, YCfg<Rad<9, 7, 14>>::SMEM_BYTES, launch_y_882_1},
    {882, 2, 7, 9, 14, YCfg<Rad<7, 9, 14>>::THREADS, YCfg<Rad<7, 9, 14>>::SMEM_BYTES, launch_y_882_2},
    {896, 0, 14, 8, 8, YCfg<Rad<14, 8, 8>>::THREADS, YCfg<Rad<14, 8, 8>>::SMEM_BYTES, launch_y_896_0},
    {896, 1, 8, 8, 14, YCfg<Rad<8, 8, 14>>::THREADS, YCfg<Rad<8, 8, 14>>::SMEM_BYTES, launch_y_896_1},
    {896, 2, 16, 7, 8, YCfg<Rad<16, 7, 8>>::THREADS, YCfg<Rad<16, 7, 8>>::SMEM_BYTES, launch_y_896_2},
    {900, 0, 10, 9, 10, YCfg<Rad<10, 9, 10>>::THREADS, YCfg<Rad<10, 9, 10>>::SMEM_BYTES, launch_y_900_0},
    {900, 1, 9, 10, 10, YCfg<Rad<9, 10, 10>>::THREADS, YCfg<Rad<9, 10, 10>>::SMEM_BYTES, launch_y_900_1},
    {900, 2, 15, 6, 10, YCfg<Rad<15, 6, 10>>::THREADS, YCfg<Rad<15, 6, 10>>::SMEM_BYTES, launch_y_900_2},
    {945, 0, 15, 7, 9, YCfg<Rad<15, 7, 9>>::THREADS, YCfg<Rad<15, 7, 9>>::SMEM_BYTES, launch_y_945_0},
    {945, 1, 9, 7, 15, YCfg<Rad<9, 7, 15>>::THREADS, YCfg<Rad<9, 7, 15>>::SMEM_BYTES, launch_y_945_1},
    {945, 2, 7, 9, 15, YCfg<Rad<7, 9, 15>>::THREADS, YCfg<Rad<7, 9, 15>>::SMEM_BYTES, launch_y_945_2},
    {960, 0, 12, 8, 10, YCfg<Rad<12, 8, 10>>::THREADS, YCfg<Rad<12, 8, 10>>::SMEM_BYTES, launch_y_960_0},
    {960, 1, 10, 8, 12, YCfg<Rad<10, 8, 12>>::THREADS, YCfg<Rad<10, 8, 12>>::SMEM_BYTES, launch_y_960_1},
    {960, 2, 8, 10, 12, YCfg<Rad<8, 10, 12>>::THREADS, YCfg<Rad<8, 10, 12>>::SMEM_BYTES, launch_y_960_2},
    {972, 0, 12, 9, 9, YCfg<Rad<12, 9, 9>>::THREADS, YCfg<Rad<12, 9, 9>>::SMEM_BYTES, launch_y_972_0},
    {972, 1, 9, 9, 12, YCfg<Rad<9, 9, 12>>::THREADS, YCfg<Rad<9, 9, 12>>::SMEM_BYTES, launch_y_972_1},
    {980, 0, 14, 7, 10, YCfg<Rad<14, 7, 10>>::THREADS, YCfg<Rad<14, 7, 10>>::SMEM_BYTES, launch_y_980_0},
    {980, 1, 10, 7, 14, YCfg<Rad<10, 7, 14>>::THREADS, YCfg<Rad<10, 7, 14>>::SMEM_BYTES, launch_y_980_1},
    {980, 2, 7, 10, 14, YCfg<Rad<7, 10, 14>>::THREADS, YCfg<Rad<7, 10, 14>>::SMEM_BYTES, launch_y_980_2},
    {1000, 0, 10, 10, 10, YCfg<Rad<10, 10, 10>>::THREADS, YCfg<Rad<10, 10, 10>>::SMEM_BYTES, launch_y_1000_0},
    {1008, 0, 14, 8, 9, YCfg<Rad<14, 8, 9>>::THREADS, YCfg<Rad<14, 8, 9>>::SMEM_BYTES, launch_y_1008_0},
    {1008, 1, 9, 8, 14, YCfg<Rad<9, 8, 14>>::THREADS, YCfg<Rad<9, 8, 14>>::SMEM_BYTES, launch_y_1008_1},
    {1008, 2, 8, 9, 14, YCfg<Rad<8, 9, 14>>::THREADS, YCfg<Rad<8, 9, 14>>::SMEM_BYTES, launch_y_1008_2},
    {1024, 0, 16, 8, 8, YCfg<Rad<16, 8, 8>>::THREADS, YCfg<Rad<16, 8, 8>>::SMEM_BYTES, launch_y_1024_0},
    {1024, 1, 8, 8, 16, YCfg<Rad<8, 8, 16>>::THREADS, YCfg<Rad<8, 8, 16>>::SMEM_BYTES, launch_y_1024_1},
    {1024, 2, 4, 16, 16, YCfg<Rad<4, 16, 16>>::THREADS, YCfg<Rad<4, 16, 16>>::SMEM_BYTES, launch_y_1024_2},
    {1050, 0, 15, 7, 10, YCfg<Rad<15, 7, 10>>::THREADS, YCfg<Rad<15, 7, 10>>::SMEM_BYTES, launch_y_1050_0},
    {1050, 1, 10, 7, 15, YCfg<Rad<10, 7, 15>>::THREADS, YCfg<Rad<10, 7, 15>>::SMEM_BYTES, launch_y_1050_1},
    {1050, 2, 7, 10, 15, YCfg<Rad<7, 10, 15>>::THREADS, YCfg<Rad<7, 10, 15>>::SMEM_BYTES, launch_y_1050_2},
    {1080, 0, 12, 9, 10, YCfg<Rad<12, 9, 10>>::THREADS, YCfg<Rad<12, 9, 10>>::SMEM_BYTES, launch_y_1080_0},
    {1080, 1, 10, 9, 12, YCfg<Rad<10, 9, 12>>::THREADS, YCfg<Rad<10, 9, 12>>::SMEM_BYTES, launch_y_1080_1},
    {1080, 2, 9, 10, 12, YCfg<Rad<9, 10, 12>>::THREADS, YCfg<Rad<9, 10, 12>>::SMEM_BYTES, launch_y_1080_2},
    {1120, 0, 14, 8, 10, YCfg<Rad<14, 8, 10>>::THREADS, YCfg<Rad<14, 8, 10>>::SMEM_BYTES, launch_y_1120_0},
    {1120, 1, 10, 8, 14, YCfg<Rad<10, 8, 14>>::THREADS, YCfg<Rad<10, 8, 14>>::SMEM_BYTES, launch_y_1120_1},
    {1120, 2, 8, 10, 14, YCfg<Rad<8, 10, 14>>::THREADS, YCfg<Rad<8, 10, 14>>::SMEM_BYTES, launch_y_1120_2},
    {1125, 0, 15, 5, 15, YCfg<Rad<15, 5, 15>>::THREADS, YCfg<Rad<15, 5, 15>>::SMEM_BYTES, launch_y_1125_0},
    {1125, 1, 5, 15, 15, YCfg<Rad<5, 15, 15>>::THREADS, YCfg<Rad<5, 15, 15>>::SMEM_BYTES, launch_y_1125_1},
    {1134, 0, 14, 9, 9, YCfg<Rad<14, 9, 9>>::THREADS, YCfg<Rad<14, 9, 9>>::SMEM_BYTES, launch_y_1134_0},
    {1134, 1, 9, 9, 14, YCfg<Rad<9, 9, 14>>::THREADS, YCfg<Rad<9, 9, 14>>::SMEM_BYTES, launch_y_1134_1},
    {1152, 0, 12, 8, 12, YCfg<Rad<12, 8, 12>>::THREADS, YCfg<Rad<12, 8, 12>>::SMEM_BYTES, launch_y_1152_0},
    {1152, 1, 8, 12, 12, YCfg<Rad<8, 12, 12>>::THREADS, YCfg<Rad<8, 12, 12>>::SMEM_BYTES, launch_y_1152_1},
    {1152, 2, 16, 8, 9, YCfg<Rad<16, 8, 9>>::THREADS, YCfg<Rad<16, 8, 9>>::SMEM_BYTES, launch_y_1152_2},
    {1176, 0, 14, 7, 12, YCfg<Rad<14, 7, 12>>::THREADS, YCfg<Rad<14, 7, 12>>::SMEM_BYTES, launch_y_1176_0},
    {1176, 1, 12, 7, 14, YCfg<Rad<12, 7, 14>>::THREADS, YCfg<Rad<12, 7, 14>>::SMEM_BYTES, launch_y_1176_1},
    {1176, 2, 7, 12, 14, YCfg<Rad<7, 12, 14>>::THREADS, YCfg<Rad<7, 12, 14>>::SMEM_BYTES, launch_y_1176_2},
    {1200, 0, 12, 10, 10, YCfg<Rad<12, 10, 10>>::THREADS, YCfg<Rad<12, 10, 10>>::SMEM_BYTES, launch_y_1200_0},
    {1200, 1, 10, 10, 12, YCfg<Rad<10, 10, 12>>::THREADS, YCfg<Rad<10, 10, 12>>::SMEM_BYTES, launch_y_1200_1},
    {1200, 2, 15, 8, 10, YCfg<Rad<15, 8, 10>>::THREADS, YCfg<Rad<15, 8, 10>>::SMEM_BYTES, launch_y_1200_2},
    {1215, 0, 15, 9, 9, YCfg<Rad<15, 9, 9>>::THREADS, YCfg<Rad<15, 9, 9>>::SMEM_BYTES, launch_y_1215_0},
    {1215, 1, 9, 9, 15, YCfg<Rad<9, 9, 15>>::THREADS, YCfg<Rad<9, 9, 15>>::SMEM_BYTES, launch_y_1215_1},
    {1260, 0, 14, 9, 10, YCfg<Rad<14, 9, 10>>::THREADS, YCfg<Rad<14, 9, 10>>::SMEM_BYTES, launch_y_1260_0},
    {1260, 1, 10, 9, 14, YCfg<Rad<10, 9, 14>>::THREADS, YCfg<Rad<10, 9, 14>>::SMEM_BYTES, launch_y_1260_1},
    {1260, 2, 9, 10, 14, YCfg<Rad<9, 10, 14>>::THREADS, YCfg<Rad<9, 10, 14>>::SMEM_BYTES, launch_y_1260_2},
    {1280, 0, 16, 8, 10, YCfg<Rad<16, 8, 10>>::THREADS, YCfg<Rad<16, 8, 10>>::SMEM_BYTES, launch_y_1280_0},
    {1280, 1, 10, 8, 16, YCfg<Rad<10, 8, 16>>::THREADS, YCfg<Rad<10, 8, 16>>::SMEM_BYTES, launch_y_1280_1},
    {1280, 2, 8, 10, 16, YCfg<Rad<8, 10, 16>>::THREADS, YCfg<Rad<8, 10, 16>>::SMEM_BYTES, launch_y_1280_2},
    {1296, 0, 12, 9, 12, YCfg<Rad<12, 9, 12>>::THREADS, YCfg<Rad<12, 9, 12>>::SMEM_BYTES, launch_y_1296_0},
    {1296, 1, 9, 12, 12, YCfg<Rad<9, 12, 12>>::THREADS, YCfg<Rad<9, 12, 12>>::SMEM_BYTES, launch_y_1296_1},
    {1296, 2, 16, 9, 9, YCfg<Rad<16, 9, 9>>::THREADS, YCfg<Rad<16, 9, 9>>::SMEM_BYTES, launch_y_1296_2},
    {1344, 0, 14, 8, 12, YCfg<Rad<14, 8, 12>>::THREADS, YCfg<Rad<14, 8, 12>>::SMEM_BYTES, launch_y_1344_0},
    {1344, 1, 12, 8, 14, YCfg<Rad<12, 8, 14>>::THREADS, YCfg<Rad<12, 8, 14>>::SMEM_BYTES, launch_y_1344_1},
    {1344, 2, 8, 12, 14, YCfg<Rad<8, 12, 14>>::THREADS, YCfg<Rad<8, 12, 14>>::SMEM_BYTES, launch_y_1344_2},
    {1350, 0, 15, 9, 10, YCfg<Rad<15, 9, 10>>::THREADS, YCfg<Rad<15, 9, 10>>::SMEM_BYTES, launch_y_1350_0},
    {1350, 1, 10, 9, 15, YCfg<Rad<10, 9, 15>>::THREADS, YCfg<Rad<10, 9, 15>>::SMEM_BYTES, launch_y_1350_1},
    {1350, 2, 9, 10, 15, YCfg<Rad<9, 10, 15>>::THREADS, YCfg<Rad<9, 10, 15>>::SMEM_BYTES, launch_y_1350_2},
    {1372, 0, 14, 7, 14, YCfg<Rad<14, 7, 14>>::THREADS, YCfg<Rad<14, 7, 14>>::SMEM_BYTES, launch_y_1372_0},
    {1372, 1, 7, 14, 14, YCfg<Rad<7, 14, 14>>::THREADS, YCfg<Rad<7, 14, 14>>::SMEM_BYTES, launch_y_1372_1},
    {1400, 0, 14, 10, 10, YCfg<Rad<14, 10, 10>>::THREADS, YCfg<Rad<14, 10, 10>>::SMEM_BYTES, launch_y_1400_0},
    {1400, 1, 10, 10, 14, YCfg<Rad<10, 10, 14>>::THREADS, YCfg<Rad<10, 10, 14>>::SMEM_BYTES, launch_y_1400_1},
    {1440, 0, 12, 10, 12, YCfg<Rad<12, 10, 12>>::THREADS, YCfg<Rad<12, 10, 12>>::SMEM_BYTES, launch_y_1440_0},
    {1440, 1, 10, 12, 12, YCfg<Rad<10, 12, 12>>::THREADS, YCfg<Rad<10, 12, 12>>::SMEM_BYTES, launch_y_1440_1},
    {1440, 2, 16, 9, 10, YCfg<Rad<16, 9, 10>>::THREADS, YCfg<Rad<16, 9, 10>>::SMEM_BYTES, launch_y_1440_2},
    {1470, 0, 15, 7, 14, YCfg<Rad<15, 7, 14>>::THREADS, YCfg<Rad<15, 7, 14>>::SMEM_BYTES, launch_y_1470_0},
    {1470, 1, 14, 7, 15, YCfg<Rad<14, 7, 15>>::THREADS, YCfg<Rad<14, 7, 15>>::SMEM_BYTES, launch_y_1470_1},
    {1470, 2, 7, 14, 15, YCfg<Rad<7, 14, 15>>::THREADS, YCfg<Rad<7, 14, 15>>::SMEM_BYTES, launch_y_1470_2},
    {1500, 0, 15, 10, 10, YCfg<Rad<15, 10, 10>>::THREADS, YCfg<Rad<15, 10, 10>>::SMEM_BYTES, launch_y_1500_0},
    {1500, 1, 10, 10, 15, YCfg<Rad<10, 10, 15>>::THREADS, YCfg<Rad<10, 10, 15>>::SMEM_BYTES, launch_y_1500_1},
    {1512, 0, 14, 9, 12, YCfg<Rad<14, 9, 12>>::THREADS, YCfg<Rad<14, 9, 12>>::SMEM_BYTES, launch_y_1512_0},
    {1512, 1, 12, 9, 14, YCfg<Rad<12, 9, 14>>::THREADS, YCfg<Rad<12, 9, 14>>::SMEM_BYTES, launch_y_1512_1},
    {1512, 2, 9, 12, 14, YCfg<Rad<9, 12, 14>>::THREADS, YCfg<Rad<9, 12, 14>>::SMEM_BYTES, launch_y_1512_2},
    {1536, 0, 16, 8, 12, YCfg<Rad<16, 8, 12>>::THREADS, YCfg<Rad<16, 8, 12>>::SMEM_BYTES, launch_y_1536_0},
    {1536, 1, 12, 8, 16, YCfg<Rad<12, 8, 16>>::THREADS, YCfg<Rad<12, 8, 16>>::SMEM_BYTES, launch_y_1536_1},
    {1536, 2, 8, 12, 16, YCfg<Rad<8, 12, 16>>::THREADS, YCfg<Rad<8, 12, 16>>::SMEM_BYTES, launch_y_1536_2},
    {1568, 0, 14, 8, 14, YCfg<Rad<14, 8, 14>>::THREADS, YCfg<Rad<14, 8, 14>>::SMEM_BYTES, launch_y_1568_0},
    {1568, 1, 8, 14, 14, YCfg<Rad<8, 14, 14>>::THREADS, YCfg<Rad<8, 14, 14>>::SMEM_BYTES, launch_y_1568_1},
    {1568, 2, 16, 7, 14, YCfg<Rad<16, 7, 14>>::THREADS, YCfg<Rad<16, 7, 14>>::SMEM_BYTES, launch_y_1568_2},
    {1575, 0, 15, 7, 15, YCfg<Rad<15, 7, 15>>::THREADS, YCfg<Rad<15, 7, 15>>::SMEM_BYTES, launch_y_1575_0},
    {1575, 1, 7, 15, 15, YCfg<Rad<7, 15, 15>>::THREADS, YCfg<Rad<7, 15, 15>>::SMEM_BYTES, launch_y_1575_1},
    {1600, 0, 16, 10, 10, YCfg<Rad<16, 10, 10>>::THREADS, YCfg<Rad<16, 10, 10>>::SMEM_BYTES, launch_y_1600_0},
    {1600, 1, 10, 10, 16, YCfg<Rad<10, 10, 16>>::THREADS, YCfg<Rad<10, 10, 16>>::SMEM_BYTES, launch_y_1600_1},
    {1620, 0, 15, 9, 12, YCfg<Rad<15, 9, 12>>::THREADS, YCfg<Rad<15, 9, 12>>::SMEM_BYTES, launch_y_1620_0},
    {1620, 1, 12, 9, 15, YCfg<Rad<12, 9, 15>>::THREADS, YCfg<Rad<12, 9, 15>>::SMEM_BYTES, launch_y_1620_1},
    {1620, 2, 9, 12, 15, YCfg<Rad<9, 12, 15>>::THREADS, YCfg<Rad<9, 12, 15>>::SMEM_BYTES, launch_y_1620_2},
    {1680, 0, 14, 10, 12, YCfg<Rad<14, 10, 12>>::THREADS, YCfg<Rad<14, 10, 12>>::SMEM_BYTES, launch_y_1680_0},
    {1680, 1, 12, 10, 14, YCfg<Rad<12, 10, 14>>::THREADS, YCfg<Rad<12, 10, 14>>::SMEM_BYTES, launch_y_1680_1},
    {1680, 2, 10, 12, 14, YCfg<Rad<10, 12, 14>>::THREADS, YCfg<Rad<10, 12, 14>>::SMEM_BYTES, launch_y_1680_2},
    {1728, 0, 12, 12, 12, YCfg<Rad<12, 12, 12>>::THREADS, YCfg<Rad<12, 12, 12>>::SMEM_BYTES, launch_y_1728_0},
    {1728, 1, 16, 9, 12, YCfg<Rad<16, 9, 12>>::THREADS, YCfg<Rad<16, 9, 12>>::SMEM_BYTES, launch_y_1728_1},
    {1728, 2, 9, 12, 16, YCfg<Rad<9, 12, 16>>::THREADS, YCfg<Rad<9, 12, 16>>::SMEM_BYTES, launch_y_1728_2},
    {1764, 0, 14, 9, 14, YCfg<Rad<14, 9, 14>>::THREADS, YCfg<Rad<14, 9, 14>>::SMEM_BYTES, launch_y_1764_0},
    {1764, 1, 9, 14, 14, YCfg<Rad<9, 14, 14>>::THREADS, YCfg<Rad<9, 14, 14>>::SMEM_BYTES, launch_y_1764_1},
    {1792, 0, 16, 8, 14, YCfg<Rad<16, 8, 14>>::THREADS, YCfg<Rad<16, 8, 14>>::SMEM_BYTES, launch_y_1792_0},
    {1792, 1, 14, 8, 16, YCfg<Rad<14, 8, 16>>::THREADS, YCfg<Rad<14, 8, 16>>::SMEM_BYTES, launch_y_1792_1},
    {1792, 2, 8, 14, 16, YCfg<Rad<8, 14, 16>>::THREADS, YCfg<Rad<8, 14, 16>>::SMEM_BYTES, launch_y_1792_2},
    {1800, 0, 15, 10, 12, YCfg<Rad<15, 10, 12>>::THREADS, YCfg<Rad<15, 10, 12>>::SMEM_BYTES, launch_y_1800_0},
    {1800, 1, 12, 10, 15, YCfg<Rad<12, 10, 15>>::THREADS, YCfg<Rad<12, 10, 15>>::SMEM_BYTES, launch_y_1800_1},
    {1800, 2, 10, 12, 15, YCfg<Rad<10, 12, 15>>::THREADS, YCfg<Rad<10, 12, 15>>::SMEM_BYTES, launch_y_1800_2},
    {1890, 0, 15, 9, 14, YCfg<Rad<15, 9, 14>>::THREADS, YCfg<Rad<15, 9, 14>>::SMEM_BYTES, launch_y_1890_0},
    {1890, 1, 14, 9, 15, YCfg<Rad<14, 9, 15>>::THREADS, YCfg<Rad<14, 9, 15>>::SMEM_BYTES, launch_y_1890_1},
    {1890, 2, 9, 14, 15, YCfg<Rad<9, 14, 15>>::THREADS, YCfg<Rad<9, 14, 15>>::SMEM_BYTES, launch_y_1890_2},
    {1920, 0, 16, 10, 12, YCfg<Rad<16, 10, 12>>::THREADS, YCfg<Rad<16, 10, 12>>::SMEM_BYTES, launch_y_1920_0},
    {1920, 1, 12, 10, 16, YCfg<Rad<12, 10, 16>>::THREADS, YCfg<Rad<12, 10, 16>>::SMEM_BYTES, launch_y_1920_1},
    {1920, 2, 10, 12, 16, YCfg<Rad<10, 12, 16>>::THREADS, YCfg<Rad<10, 12, 16>>::SMEM_BYTES, launch_y_1920_2},
    {1960, 0, 14, 10, 14, YCfg<Rad<14, 10, 14>>::THREADS, YCfg<Rad<14, 10, 14>>::SMEM_BYTES, launch_y_1960_0},
    {1960, 1, 10, 14, 14, YCfg<Rad<10, 14, 14>>::THREADS, YCfg<Rad<10, 14, 14>>::SMEM_BYTES, launch_y_1960_1},
    {2016, 0, 14, 12, 12, YCfg<Rad<14, 12, 12>>::THREADS, YCfg<Rad<14, 12, 12>>::SMEM_BYTES, launch_y_2016_0},
    {2016, 1, 12, 12, 14, YCfg<Rad<12, 12, 14>>::THREADS, YCfg<Rad<12, 12, 14>>::SMEM_BYTES, launch_y_2016_1},
    {2016, 2, 16, 9, 14, YCfg<Rad<16, 9, 14>>::THREADS, YCfg<Rad<16, 9, 14>>::SMEM_BYTES, launch_y_2016_2},
    {2025, 0, 15, 9, 15, YCfg<Rad<15, 9, 15>>::THREADS, YCfg<Rad<15, 9, 15>>::SMEM_BYTES, launch_y_2025_0},
    {2025, 1, 9, 15, 15, YCfg<Rad<9, 15, 15>>::THREADS, YCfg<Rad<9, 15, 15>>::SMEM_BYTES, launch_y_2025_1},
    {2048, 0, 16, 8, 16, YCfg<Rad<16, 8, 16>>::THREADS, YCfg<Rad<16, 8, 16>>::SMEM_BYTES, launch_y_2048_0},
    {2048, 1, 8, 16, 16, YCfg<Rad<8, 16, 16>>::THREADS, YCfg<Rad<8, 16, 16>>::SMEM_BYTES, launch_y_2048_1},
    {2100, 0, 15, 10, 14, YCfg<Rad<15, 10, 14>>::THREADS, YCfg<Rad<15, 10, 14>>::SMEM_BYTES, launch_y_2100_0},
    {2100, 1, 14, 10, 15, YCfg<Rad<14, 10, 15>>::THREADS, YCfg<Rad<14, 10, 15>>::SMEM_BYTES, launch_y_2100_1},
    {2100, 2, 10, 14, 15, YCfg<Rad<10, 14, 15>>::THREADS, YCfg<Rad<10, 14, 15>>::SMEM_BYTES, launch_y_2100_2},
    {2160, 0, 15, 12, 12, YCfg<Rad<15, 12, 12>>::THREADS, YCfg<Rad<15, 12, 12>>::SMEM_BYTES, launch_y_2160_0},
    {2160, 1, 12, 12, 15, YCfg<Rad<12, 12, 15>>::THREADS, YCfg<Rad<12, 12, 15>>::SMEM_BYTES, launch_y_2160_1},
    {2160, 2, 16, 9, 15, YCfg<Rad<16, 9, 15>>::THREADS, YCfg<Rad<16, 9, 15>>::SMEM_BYTES, launch_y_2160_2},
    {2240, 0, 16, 10, 14, YCfg<Rad<16, 10, 14>>::THREADS, YCfg<Rad<16, 10, 14>>::SMEM_BYTES, launch_y_2240_0},
    {2240, 1, 14, 10, 16, YCfg<Rad<14, 10, 16>>::THREADS, YCfg<Rad<14, 10, 16>>::SMEM_BYTES, launch_y_2240_1},
    {2240, 2, 10, 14, 16, YCfg<Rad<10, 14, 16>>::THREADS, YCfg<Rad<10, 14, 16>>::SMEM_BYTES, launch_y_2240_2},
    {2250, 0, 15, 10, 15, YCfg<Rad<15, 10, 15>>::THREADS, YCfg<Rad<15, 10, 15>>::SMEM_BYTES, launch_y_2250_0},
    {2250, 1, 10, 15, 15, YCfg<Rad<10, 15, 15>>::THREADS, YCfg<Rad<10, 15, 15>>::SMEM_BYTES, launch_y_2250_1},
    {2304, 0, 16, 12, 12, YCfg<Rad<16, 12, 12>>::THREADS, YCfg<Rad<16, 12, 12>>::SMEM_BYTES, launch_y_2304_0},
    {2304, 1, 12, 12, 16, YCfg<Rad<12, 12, 16>>::THREADS, YCfg<Rad<12, 12, 16>>::SMEM_BYTES, launch_y_2304_1},
    {2304, 2, 9, 16, 16, YCfg<Rad<9, 16, 16>>::THREADS, YCfg<Rad<9, 16, 16>>::SMEM_BYTES, launch_y_2304_2},
    {2352, 0, 14, 12, 14, YCfg<Rad<14, 12, 14>>::THREADS, YCfg<Rad<14, 12, 14>>::SMEM_BYTES, launch_y_2352_0},
    {2352, 1, 12, 14, 14, YCfg<Rad<12, 14, 14>>::THREADS, YCfg<Rad<12, 14, 14>>::SMEM_BYTES, launch_y_2352_1},
    {2400, 0, 16, 10, 15, YCfg<Rad<16, 10, 15>>::THREADS, YCfg<Rad<16, 10, 15>>::SMEM_BYTES, launch_y_2400_0},
    {2400, 1, 15, 10, 16, YCfg<Rad<15, 10, 16>>::THREADS, YCfg<Rad<15, 10, 16>>::SMEM_BYTES, launch_y_2400_1},
    {2400, 2, 10, 15, 16, YCfg<Rad<10, 15, 16>>::THREADS, YCfg<Rad<10, 15, 16>>::SMEM_BYTES, launch_y_2400_2},
    {2520, 0, 15, 12, 14, YCfg<Rad<15, 12, 14>>::THREADS, YCfg<Rad<15, 12, 14>>::SMEM_BYTES, launch_y_2520_0},
    {2520, 1, 14, 12, 15, YCfg<Rad<14, 12, 15>>::THREADS, YCfg<Rad<14, 12, 15>>::SMEM_BYTES, launch_y_2520_1},
    {2520, 2, 12, 14, 15, YCfg<Rad<12, 14, 15>>::THREADS, YCfg<Rad<12, 14, 15>>::SMEM_BYTES, launch_y_2520_2},
    {2560, 0, 16, 10, 16, YCfg<Rad<16, 10, 16>>::THREADS, YCfg<Rad<16, 10, 16>>::SMEM_BYTES, launch_y_2560_0},
    {2560, 1, 10, 16, 16, YCfg<Rad<10, 16, 16>>::THREADS, YCfg<Rad<10, 16, 16>>::SMEM_BYTES, launch_y_2560_1},
    {2688, 0, 16, 12, 14, YCfg<Rad<16, 12, 14>>::THREADS, YCfg<Rad<16, 12, 14>>::SMEM_BYTES, launch_y_2688_0},
    {2688, 1, 14, 12, 16, YCfg<Rad<14, 12, 16>>::THREADS, YCfg<Rad<14, 12, 16>>::SMEM_BYTES, launch_y_2688_1},
    {2688, 2, 12, 14, 16, YCfg<Rad<12, 14, 16>>::THREADS, YCfg<Rad<12, 14, 16>>::SMEM_BYTES, launch_y_2688_2},
    {2700, 0, 15, 12, 15, YCfg<Rad<15, 12, 15>>::THREADS, YCfg<Rad<15, 12, 15>>::SMEM_BYTES, launch_y_2700_0},
    {2700, 1, 12, 15, 15, YCfg<Rad<12, 15, 15>>::THREADS, YCfg<Rad<12, 15, 15>>::SMEM_BYTES, launch_y_2700_1},
    {2744, 0, 14, 14, 14, YCfg<Rad<14, 14, 14>>::THREADS, YCfg<Rad<14, 14, 14>>::SMEM_BYTES, launch_y_2744_0},
    {2880, 0, 16, 12, 15, YCfg<Rad<16, 12, 15>>::THREADS, YCfg<Rad<16, 12, 15>>::SMEM_BYTES, launch_y_2880_0},
    {2880, 1, 15, 12, 16, YCfg<Rad<15, 12, 16>>::THREADS, YCfg<Rad<15, 12, 16>>::SMEM_BYTES, launch_y_2880_1},
    {2880, 2, 12, 15, 16, YCfg<Rad<12, 15, 16>>::THREADS, YCfg<Rad<12, 15, 16>>::SMEM_BYTES, launch_y_2880_2},
    {2940, 0, 15, 14, 14, YCfg<Rad<15, 14, 14>>::THREADS, YCfg<Rad<15, 14, 14>>::SMEM_BYTES, launch_y_2940_0},
    {2940, 1, 14, 14, 15, YCfg<Rad<14, 14, 15>>::THREADS, YCfg<Rad<14, 14, 15>>::SMEM_BYTES, launch_y_2940_1},
    {3072, 0, 16, 12, 16, YCfg<Rad<16, 12, 16>>::THREADS, YCfg<Rad<16, 12, 16>>::SMEM_BYTES, launch_y_3072_0},
    {3072, 1, 12, 16, 16, YCfg<Rad<12, 16, 16>>::THREADS, YCfg<Rad<12, 16, 16>>::SMEM_BYTES, launch_y_3072_1},
    {3136, 0, 16, 14, 14, YCfg<Rad<16, 14, 14>>::THREADS, YCfg<Rad<16, 14, 14>>::SMEM_BYTES, launch_y_3136_0},
    {3136, 1, 14, 14, 16, YCfg<Rad<14, 14, 16>>::THREADS, YCfg<Rad<14, 14, 16>>::SMEM_BYTES, launch_y_3136_1},
    {3150, 0, 15, 14, 15, YCfg<Rad<15, 14, 15>>::THREADS, YCfg<Rad<15, 14, 15>>::SMEM_BYTES, launch_y_3150_0},
    {3150, 1, 14, 15, 15, YCfg<Rad<14, 15, 15>>::THREADS, YCfg<Rad<14, 15, 15>>::SMEM_BYTES, launch_y_3150_1},
};
}  // namespace dwcu
