// generated by gen_plans.py -- do not edit
#pragma once
#include "passes.cuh"
namespace dwcu {
struct LinesPlan { int n, ra, rb, rc, T, threads; size_t smem; void (*launch)(const LinesArgs &, int, cudaStream_t); };
struct XPlan { int n, ra, rb, rc, R, threads; size_t smem; void (*launch)(const XArgs &, cudaStream_t); };
struct YPlan { int n, ra, rb, rc, threads; size_t smem; void (*launch)(const YArgs &, cudaStream_t); };
void launch_lines_1(const LinesArgs &, int, cudaStream_t);
void launch_lines_2(const LinesArgs &, int, cudaStream_t);
void launch_lines_3(const LinesArgs &, int, cudaStream_t);
void launch_lines_4(const LinesArgs &, int, cudaStream_t);
void launch_lines_5(const LinesArgs &, int, cudaStream_t);
void launch_lines_6(const LinesArgs &, int, cudaStream_t);
void launch_lines_7(const LinesArgs &, int, cudaStream_t);
void launch_lines_8(const LinesArgs &, int, cudaStream_t);
void launch_lines_9(const LinesArgs &, int, cudaStream_t);
void launch_lines_10(const LinesArgs &, int, cudaStream_t);
void launch_lines_12(const LinesArgs &, int, cudaStream_t);
void launch_lines_14(const LinesArgs &, int, cudaStream_t);
void launch_lines_15(const LinesArgs &, int, cudaStream_t);
void launch_lines_16(const LinesArgs &, int, cudaStream_t);
void launch_lines_18(const LinesArgs &, int, cudaStream_t);
void launch_lines_20(const LinesArgs &, int, cudaStream_t);
void launch_lines_21(const LinesArgs &, int, cudaStream_t);
void launch_lines_24(const LinesArgs &, int, cudaStream_t);
void launch_lines_25(const LinesArgs &, int, cudaStream_t);
void launch_lines_27(const LinesArgs &, int, cudaStream_t);
void launch_lines_28(const LinesArgs &, int, cudaStream_t);
void launch_lines_30(const LinesArgs &, int, cudaStream_t);
void launch_lines_32(const LinesArgs &, int, cudaStream_t);
void launch_lines_35(const LinesArgs &, int, cudaStream_t);
void launch_lines_36(const LinesArgs &, int, cudaStream_t);
void launch_lines_40(const LinesArgs &, int, cudaStream_t);
void launch_lines_42(const LinesArgs &, int, cudaStream_t);
void launch_lines_45(const LinesArgs &, int, cudaStream_t);
void launch_lines_48(const LinesArgs &, int, cudaStream_t);
void launch_lines_49(const LinesArgs &, int, cudaStream_t);
void launch_lines_50(const LinesArgs &, int, cudaStream_t);
void launch_lines_54(const LinesArgs &, int, cudaStream_t);
void launch_lines_56(const LinesArgs &, int, cudaStream_t);
void launch_lines_60(const LinesArgs &, int, cudaStream_t);
void launch_lines_63(const LinesArgs &, int, cudaStream_t);
void launch_lines_64(const LinesArgs &, int, cudaStream_t);
void launch_lines_70(const LinesArgs &, int, cudaStream_t);
void launch_lines_72(const LinesArgs &, int, cudaStream_t);
void launch_lines_75(const LinesArgs &, int, cudaStream_t);
void launch_lines_80(const LinesArgs &, int, cudaStream_t);
void launch_lines_81(const LinesArgs &, int, cudaStream_t);
void launch_lines_84(const LinesArgs &, int, cudaStream_t);
void launch_lines_90(const LinesArgs &, int, cudaStream_t);
void launch_lines_96(const LinesArgs &, int, cudaStream_t);
void launch_lines_98(const LinesArgs &, int, cudaStream_t);
void launch_lines_100(const LinesArgs &, int, cudaStream_t);
void launch_lines_105(const LinesArgs &, int, cudaStream_t);
void launch_lines_108(const LinesArgs &, int, cudaStream_t);
void launch_lines_112(const LinesArgs &, int, cudaStream_t);
void launch_lines_120(const LinesArgs &, int, cudaStream_t);
void launch_lines_125(const LinesArgs &, int, cudaStream_t);
void launch_lines_126(const LinesArgs &, int, cudaStream_t);
void launch_lines_128(const LinesArgs &, int, cudaStream_t);
void launch_lines_135(const LinesArgs &, int, cudaStream_t);
void launch_lines_140(const LinesArgs &, int, cudaStream_t);
void launch_lines_144(const LinesArgs &, int, cudaStream_t);
void launch_lines_147(const LinesArgs &, int, cudaStream_t);
void launch_lines_150(const LinesArgs &, int, cudaStream_t);
void launch_lines_160(const LinesArgs &, int, cudaStream_t);
void launch_lines_162(const LinesArgs &, int, cudaStream_t);
void launch_lines_168(const LinesArgs &, int, cudaStream_t);
void launch_lines_175(const LinesArgs &, int, cudaStream_t);
void launch_lines_180(const LinesArgs &, int, cudaStream_t);
void launch_lines_189(const LinesArgs &, int, cudaStream_t);
void launch_lines_192(const LinesArgs &, int, cudaStream_t);
void launch_lines_196(const LinesArgs &, int, cudaStream_t);
void launch_lines_200(const LinesArgs &, int, cudaStream_t);
void launch_lines_210(const LinesArgs &, int, cudaStream_t);
void launch_lines_216(const LinesArgs &, int, cudaStream_t);
void launch_lines_224(const LinesArgs &, int, cudaStream_t);
void launch_lines_225(const LinesArgs &, int, cudaStream_t);
void launch_lines_240(const LinesArgs &, int, cudaStream_t);
void launch_lines_243(const LinesArgs &, int, cudaStream_t);
void launch_lines_245(const LinesArgs &, int, cudaStream_t);
void launch_lines_250(const LinesArgs &, int, cudaStream_t);
void launch_lines_252(const LinesArgs &, int, cudaStream_t);
void launch_lines_256(const LinesArgs &, int, cudaStream_t);
void launch_lines_270(const LinesArgs &, int, cudaStream_t);
void launch_lines_280(const LinesArgs &, int, cudaStream_t);
void launch_lines_288(const LinesArgs &, int, cudaStream_t);
void launch_lines_294(const LinesArgs &, int, cudaStream_t);
void launch_lines_300(const LinesArgs &, int, cudaStream_t);
void launch_lines_315(const LinesArgs &, int, cudaStream_t);
void launch_lines_320(const LinesArgs &, int, cudaStream_t);
void launch_lines_324(const LinesArgs &, int, cudaStream_t);
void launch_lines_336(const LinesArgs &, int, cudaStream_t);
void launch_lines_343(const LinesArgs &, int, cudaStream_t);
void launch_lines_350(const LinesArgs &, int, cudaStream_t);
void launch_lines_360(const LinesArgs &, int, cudaStream_t);
void launch_lines_375(const LinesArgs &, int, cudaStream_t);
void launch_lines_378(const LinesArgs &, int, cudaStream_t);
void launch_lines_384(const LinesArgs &, int, cudaStream_t);
void launch_lines_392(const LinesArgs &, int, cudaStream_t);
void launch_lines_400(const LinesArgs &, int, cudaStream_t);
void launch_lines_405(const LinesArgs &, int, cudaStream_t);
void launch_lines_420(const LinesArgs &, int, cudaStream_t);
void launch_lines_432(const LinesArgs &, int, cudaStream_t);
void launch_lines_441(const LinesArgs &, int, cudaStream_t);
void launch_lines_448(const LinesArgs &, int, cudaStream_t);
void launch_lines_450(const LinesArgs &, int, cudaStream_t);
void launch_lines_480(const LinesArgs &, int, cudaStream_t);
void launch_lines_486(const LinesArgs &, int, cudaStream_t);
void launch_lines_490(const LinesArgs &, int, cudaStream_t);
void launch_lines_500(const LinesArgs &, int, cudaStream_t);
void launch_lines_504(const LinesArgs &, int, cudaStream_t);
void launch_lines_512(const LinesArgs &, int, cudaStream_t);
void launch_lines_525(const LinesArgs &, int, cudaStream_t);
void launch_lines_540(const LinesArgs &, int, cudaStream_t);
void launch_lines_560(const LinesArgs &, int, cudaStream_t);
void launch_lines_567(const LinesArgs &, int, cudaStream_t);
void launch_lines_576(const LinesArgs &, int, cudaStream_t);
void launch_lines_588(const LinesArgs &, int, cudaStream_t);
void launch_lines_600(const LinesArgs &, int, cudaStream_t);
void launch_lines_630(const LinesArgs &, int, cudaStream_t);
void launch_lines_640(const LinesArgs &, int, cudaStream_t);
void launch_lines_648(const LinesArgs &, int, cudaStream_t);
void launch_lines_672(const LinesArgs &, int, cudaStream_t);
void launch_lines_675(const LinesArgs &, int, cudaStream_t);
void launch_lines_686(const LinesArgs &, int, cudaStream_t);
void launch_lines_700(const LinesArgs &, int, cudaStream_t);
void launch_lines_720(const LinesArgs &, int, cudaStream_t);
void launch_lines_729(const LinesArgs &, int, cudaStream_t);
void launch_lines_735(const LinesArgs &, int, cudaStream_t);
void launch_lines_750(const LinesArgs &, int, cudaStream_t);
void launch_lines_756(const LinesArgs &, int, cudaStream_t);
void launch_lines_768(const LinesArgs &, int, cudaStream_t);
void launch_lines_784(const LinesArgs &, int, cudaStream_t);
void launch_lines_800(const LinesArgs &, int, cudaStream_t);
void launch_lines_810(const LinesArgs &, int, cudaStream_t);
void launch_lines_840(const LinesArgs &, int, cudaStream_t);
void launch_lines_864(const LinesArgs &, int, cudaStream_t);
void launch_lines_882(const LinesArgs &, int, cudaStream_t);
void launch_lines_896(const LinesArgs &, int, cudaStream_t);
void launch_lines_900(const LinesArgs &, int, cudaStream_t);
void launch_lines_945(const LinesArgs &, int, cudaStream_t);
void launch_lines_960(const LinesArgs &, int, cudaStream_t);
void launch_lines_972(const LinesArgs &, int, cudaStream_t);
void launch_lines_980(const LinesArgs &, int, cudaStream_t);
void launch_lines_1000(const LinesArgs &, int, cudaStream_t);
void launch_lines_1008(const LinesArgs &, int, cudaStream_t);
void launch_lines_1024(const LinesArgs &, int, cudaStream_t);
void launch_lines_1050(const LinesArgs &, int, cudaStream_t);
void launch_lines_1080(const LinesArgs &, int, cudaStream_t);
void launch_lines_1120(const LinesArgs &, int, cudaStream_t);
void launch_lines_1125(const LinesArgs &, int, cudaStream_t);
void launch_lines_1134(const LinesArgs &, int, cudaStream_t);
void launch_lines_1152(const LinesArgs &, int, cudaStream_t);
void launch_lines_1176(const LinesArgs &, int, cudaStream_t);
void launch_lines_1200(const LinesArgs &, int, cudaStream_t);
void launch_lines_1215(const LinesArgs &, int, cudaStream_t);
void launch_lines_1260(const LinesArgs &, int, cudaStream_t);
void launch_lines_1280(const LinesArgs &, int, cudaStream_t);
void launch_lines_1296(const LinesArgs &, int, cudaStream_t);
void launch_lines_1344(const LinesArgs &, int, cudaStream_t);
void launch_lines_1350(const LinesArgs &, int, cudaStream_t);
void launch_lines_1372(const LinesArgs &, int, cudaStream_t);
void launch_lines_1400(const LinesArgs &, int, cudaStream_t);
void launch_lines_1440(const LinesArgs &, int, cudaStream_t);
void launch_lines_1470(const LinesArgs &, int, cudaStream_t);
void launch_lines_1500(const LinesArgs &, int, cudaStream_t);
void launch_lines_1512(const LinesArgs &, int, cudaStream_t);
void launch_lines_1536(const LinesArgs &, int, cudaStream_t);
void launch_lines_1568(const LinesArgs &, int, cudaStream_t);
void launch_lines_1575(const LinesArgs &, int, cudaStream_t);
void launch_lines_1600(const LinesArgs &, int, cudaStream_t);
void launch_lines_1620(const LinesArgs &, int, cudaStream_t);
void launch_lines_1680(const LinesArgs &, int, cudaStream_t);
void launch_lines_1728(const LinesArgs &, int, cudaStream_t);
void launch_lines_1764(const LinesArgs &, int, cudaStream_t);
void launch_lines_1792(const LinesArgs &, int, cudaStream_t);
void launch_lines_1800(const LinesArgs &, int, cudaStream_t);
void launch_lines_1890(const LinesArgs &, int, cudaStream_t);
void launch_lines_1920(const LinesArgs &, int, cudaStream_t);
void launch_lines_1960(const LinesArgs &, int, cudaStream_t);
void launch_lines_2016(const LinesArgs &, int, cudaStream_t);
void launch_lines_2025(const LinesArgs &, int, cudaStream_t);
void launch_lines_2048(const LinesArgs &, int, cudaStream_t);
void launch_lines_2100(const LinesArgs &, int, cudaStream_t);
void launch_lines_2160(const LinesArgs &, int, cudaStream_t);
void launch_lines_2240(const LinesArgs &, int, cudaStream_t);
void launch_lines_2250(const LinesArgs &, int, cudaStream_t);
void launch_lines_2304(const LinesArgs &, int, cudaStream_t);
void launch_lines_2352(const LinesArgs &, int, cudaStream_t);
void launch_lines_2400(const LinesArgs &, int, cudaStream_t);
void launch_lines_2520(const LinesArgs &, int, cudaStream_t);
void launch_lines_2560(const LinesArgs &, int, cudaStream_t);
void launch_lines_2688(const LinesArgs &, int, cudaStream_t);
void launch_lines_2700(const LinesArgs &, int, cudaStream_t);
void launch_lines_2744(const LinesArgs &, int, cudaStream_t);
void launch_lines_2880(const LinesArgs &, int, cudaStream_t);
void launch_lines_2940(const LinesArgs &, int, cudaStream_t);
void launch_lines_3072(const LinesArgs &, int, cudaStream_t);
void launch_lines_3136(const LinesArgs &, int, cudaStream_t);
void launch_lines_3150(const LinesArgs &, int, cudaStream_t);
void launch_lines_3360(const LinesArgs &, int, cudaStream_t);
void launch_lines_3375(const LinesArgs &, int, cudaStream_t);
void launch_lines_3584(const LinesArgs &, int, cudaStream_t);
void launch_lines_3600(const LinesArgs &, int, cudaStream_t);
void launch_lines_3840(const LinesArgs &, int, cudaStream_t);
void launch_lines_4096(const LinesArgs &, int, cudaStream_t);
void launch_x_2(const XArgs &, cudaStream_t);
void launch_x_3(const XArgs &, cudaStream_t);
void launch_x_4(const XArgs &, cudaStream_t);
void launch_x_5(const XArgs &, cudaStream_t);
void launch_x_6(const XArgs &, cudaStream_t);
void launch_x_7(const XArgs &, cudaStream_t);
void launch_x_8(const XArgs &, cudaStream_t);
void launch_x_9(const XArgs &, cudaStream_t);
void launch_x_10(const XArgs &, cudaStream_t);
void launch_x_12(const XArgs &, cudaStream_t);
void launch_x_14(const XArgs &, cudaStream_t);
void launch_x_15(const XArgs &, cudaStream_t);
void launch_x_16(const XArgs &, cudaStream_t);
void launch_x_18(const XArgs &, cudaStream_t);
void launch_x_20(const XArgs &, cudaStream_t);
void launch_x_21(const XArgs &, cudaStream_t);
void launch_x_24(const XArgs &, cudaStream_t);
void launch_x_25(const XArgs &, cudaStream_t);
void launch_x_27(const XArgs &, cudaStream_t);
void launch_x_28(const XArgs &, cudaStream_t);
void launch_x_30(const XArgs &, cudaStream_t);
void launch_x_32(const XArgs &, cudaStream_t);
void launch_x_35(const XArgs &, cudaStream_t);
void launch_x_36(const XArgs &, cudaStream_t);
void launch_x_40(const XArgs &, cudaStream_t);
void launch_x_42(const XArgs &, cudaStream_t);
void launch_x_45(const XArgs &, cudaStream_t);
void launch_x_48(const XArgs &, cudaStream_t);
void launch_x_49(const XArgs &, cudaStream_t);
void launch_x_50(const XArgs &, cudaStream_t);
void launch_x_54(const XArgs &, cudaStream_t);
void launch_x_56(const XArgs &, cudaStream_t);
void launch_x_60(const XArgs &, cudaStream_t);
void launch_x_63(const XArgs &, cudaStream_t);
void launch_x_64(const XArgs &, cudaStream_t);
void launch_x_70(const XArgs &, cudaStream_t);
void launch_x_72(const XArgs &, cudaStream_t);
void launch_x_75(const XArgs &, cudaStream_t);
void launch_x_80(const XArgs &, cudaStream_t);
void launch_x_81(const XArgs &, cudaStream_t);
void launch_x_84(const XArgs &, cudaStream_t);
void launch_x_90(const XArgs &, cudaStream_t);
void launch_x_96(const XArgs &, cudaStream_t);
void launch_x_98(const XArgs &, cudaStream_t);
void launch_x_100(const XArgs &, cudaStream_t);
void launch_x_105(const XArgs &, cudaStream_t);
void launch_x_108(const XArgs &, cudaStream_t);
void launch_x_112(const XArgs &, cudaStream_t);
void launch_x_120(const XArgs &, cudaStream_t);
void launch_x_125(const XArgs &, cudaStream_t);
void launch_x_126(const XArgs &, cudaStream_t);
void launch_x_128(const XArgs &, cudaStream_t);
void launch_x_135(const XArgs &, cudaStream_t);
void launch_x_140(const XArgs &, cudaStream_t);
void launch_x_144(const XArgs &, cudaStream_t);
void launch_x_147(const XArgs &, cudaStream_t);
void launch_x_150(const XArgs &, cudaStream_t);
void launch_x_160(const XArgs &, cudaStream_t);
void launch_x_162(const XArgs &, cudaStream_t);
void launch_x_168(const XArgs &, cudaStream_t);
void launch_x_175(const XArgs &, cudaStream_t);
void launch_x_180(const XArgs &, cudaStream_t);
void launch_x_189(const XArgs &, cudaStream_t);
void launch_x_192(const XArgs &, cudaStream_t);
void launch_x_196(const XArgs &, cudaStream_t);
void launch_x_200(const XArgs &, cudaStream_t);
void launch_x_210(const XArgs &, cudaStream_t);
void launch_x_216(const XArgs &, cudaStream_t);
void launch_x_224(const XArgs &, cudaStream_t);
void launch_x_225(const XArgs &, cudaStream_t);
void launch_x_240(const XArgs &, cudaStream_t);
void launch_x_243(const XArgs &, cudaStream_t);
void launch_x_245(const XArgs &, cudaStream_t);
void launch_x_250(const XArgs &, cudaStream_t);
void launch_x_252(const XArgs &, cudaStream_t);
void launch_x_256(const XArgs &, cudaStream_t);
void launch_x_270(const XArgs &, cudaStream_t);
void launch_x_280(const XArgs &, cudaStream_t);
void launch_x_288(const XArgs &, cudaStream_t);
void launch_x_294(const XArgs &, cudaStream_t);
void launch_x_300(const XArgs &, cudaStream_t);
void launch_x_315(const XArgs &, cudaStream_t);
void launch_x_320(const XArgs &, cudaStream_t);
void launch_x_324(const XArgs &, cudaStream_t);
void launch_x_336(const XArgs &, cudaStream_t);
void launch_x_343(const XArgs &, cudaStream_t);
void launch_x_350(const XArgs &, cudaStream_t);
void launch_x_360(const XArgs &, cudaStream_t);
void launch_x_375(const XArgs &, cudaStream_t);
void launch_x_378(const XArgs &, cudaStream_t);
void launch_x_384(const XArgs &, cudaStream_t);
void launch_x_392(const XArgs &, cudaStream_t);
void launch_x_400(const XArgs &, cudaStream_t);
void launch_x_405(const XArgs &, cudaStream_t);
void launch_x_420(const XArgs &, cudaStream_t);
void launch_x_432(const XArgs &, cudaStream_t);
void launch_x_441(const XArgs &, cudaStream_t);
void launch_x_448(const XArgs &, cudaStream_t);
void launch_x_450(const XArgs &, cudaStream_t);
void launch_x_480(const XArgs &, cudaStream_t);
void launch_x_486(const XArgs &, cudaStream_t);
void launch_x_490(const XArgs &, cudaStream_t);
void launch_x_500(const XArgs &, cudaStream_t);
void launch_x_504(const XArgs &, cudaStream_t);
void launch_x_512(const XArgs &, cudaStream_t);
void launch_x_525(const XArgs &, cudaStream_t);
void launch_x_540(const XArgs &, cudaStream_t);
void launch_x_560(const XArgs &, cudaStream_t);
void launch_x_567(const XArgs &, cudaStream_t);
void launch_x_576(const XArgs &, cudaStream_t);
void launch_x_588(const XArgs &, cudaStream_t);
void launch_x_600(const XArgs &, cudaStream_t);
void launch_x_630(const XArgs &, cudaStream_t);
void launch_x_640(const XArgs &, cudaStream_t);
void launch_x_648(const XArgs &, cudaStream_t);
void launch_x_672(const XArgs &, cudaStream_t);
void launch_x_675(const XArgs &, cudaStream_t);
void launch_x_686(const XArgs &, cudaStream_t);
void launch_x_700(const XArgs &, cudaStream_t);
void launch_x_720(const XArgs &, cudaStream_t);
void launch_x_729(const XArgs &, cudaStream_t);
void launch_x_735(const XArgs &, cudaStream_t);
void launch_x_750(const XArgs &, cudaStream_t);
void launch_x_756(const XArgs &, cudaStream_t);
void launch_x_768(const XArgs &, cudaStream_t);
void launch_x_784(const XArgs &, cudaStream_t);
void launch_x_800(const XArgs &, cudaStream_t);
void launch_x_810(const XArgs &, cudaStream_t);
void launch_x_840(const XArgs &, cudaStream_t);
void launch_x_864(const XArgs &, cudaStream_t);
void launch_x_882(const XArgs &, cudaStream_t);
void launch_x_896(const XArgs &, cudaStream_t);
void launch_x_900(const XArgs &, cudaStream_t);
void launch_x_945(const XArgs &, cudaStream_t);
void launch_x_960(const XArgs &, cudaStream_t);
void launch_x_972(const XArgs &, cudaStream_t);
void launch_x_980(const XArgs &, cudaStream_t);
void launch_x_1000(const XArgs &, cudaStream_t);
void launch_x_1008(const XArgs &, cudaStream_t);
void launch_x_1024(const XArgs &, cudaStream_t);
void launch_x_1050(const XArgs &, cudaStream_t);
void launch_x_1080(const XArgs &, cudaStream_t);
void launch_x_1120(const XArgs &, cudaStream_t);
void launch_x_1125(const XArgs &, cudaStream_t);
void launch_x_1134(const XArgs &, cudaStream_t);
void launch_x_1152(const XArgs &, cudaStream_t);
void launch_x_1176(const XArgs &, cudaStream_t);
void launch_x_1200(const XArgs &, cudaStream_t);
void launch_x_1215(const XArgs &, cudaStream_t);
void launch_x_1260(const XArgs &, cudaStream_t);
void launch_x_1280(const XArgs &, cudaStream_t);
void launch_x_1296(const XArgs &, cudaStream_t);
void launch_x_1344(const XArgs &, cudaStream_t);
void launch_x_1350(const XArgs &, cudaStream_t);
void launch_x_1372(const XArgs &, cudaStream_t);
void launch_x_1400(const XArgs &, cudaStream_t);
void launch_x_1440(const XArgs &, cudaStream_t);
void launch_x_1470(const XArgs &, cudaStream_t);
void launch_x_1500(const XArgs &, cudaStream_t);
void launch_x_1512(const XArgs &, cudaStream_t);
void launch_x_1536(const XArgs &, cudaStream_t);
void launch_x_1568(const XArgs &, cudaStream_t);
void launch_x_1575(const XArgs &, cudaStream_t);
void launch_x_1600(const XArgs &, cudaStream_t);
void launch_x_1620(const XArgs &, cudaStream_t);
void launch_x_1680(const XArgs &, cudaStream_t);
void launch_x_1728(const XArgs &, cudaStream_t);
void launch_x_1764(const XArgs &, cudaStream_t);
void launch_x_1792(const XArgs &, cudaStream_t);
void launch_x_1800(const XArgs &, cudaStream_t);
void launch_x_1890(const XArgs &, cudaStream_t);
void launch_x_1920(const XArgs &, cudaStream_t);
void launch_x_1960(const XArgs &, cudaStream_t);
void launch_x_2016(const XArgs &, cudaStream_t);
void launch_x_2025(const XArgs &, cudaStream_t);
void launch_x_2048(const XArgs &, cudaStream_t);
void launch_y_2(const YArgs &, cudaStream_t);
void launch_y_3(const YArgs &, cudaStream_t);
void launch_y_4(const YArgs &, cudaStream_t);
void launch_y_5(const YArgs &, cudaStream_t);
void launch_y_6(const YArgs &, cudaStream_t);
void launch_y_7(const YArgs &, cudaStream_t);
void launch_y_8(const YArgs &, cudaStream_t);
void launch_y_9(const YArgs &, cudaStream_t);
void launch_y_10(const YArgs &, cudaStream_t);
void launch_y_12(const YArgs &, cudaStream_t);
void launch_y_14(const YArgs &, cudaStream_t);
void launch_y_15(const YArgs &, cudaStream_t);
void launch_y_16(const YArgs &, cudaStream_t);
void launch_y_18(const YArgs &, cudaStream_t);
void launch_y_20(const YArgs &, cudaStream_t);
void launch_y_21(const YArgs &, cudaStream_t);
void launch_y_24(const YArgs &, cudaStream_t);
void launch_y_25(const YArgs &, cudaStream_t);
void launch_y_27(const YArgs &, cudaStream_t);
void launch_y_28(const YArgs &, cudaStream_t);
void launch_y_30(const YArgs &, cudaStream_t);
void launch_y_32(const YArgs &, cudaStream_t);
void launch_y_35(const YArgs &, cudaStream_t);
void launch_y_36(const YArgs &, cudaStream_t);
void launch_y_40(const YArgs &, cudaStream_t);
void launch_y_42(const YArgs &, cudaStream_t);
void launch_y_45(const YArgs &, cudaStream_t);
void launch_y_48(const YArgs &, cudaStream_t);
void launch_y_49(const YArgs &, cudaStream_t);
void launch_y_50(const YArgs &, cudaStream_t);
void launch_y_54(const YArgs &, cudaStream_t);
void launch_y_56(const YArgs &, cudaStream_t);
void launch_y_60(const YArgs &, cudaStream_t);
void launch_y_63(const YArgs &, cudaStream_t);
void launch_y_64(const YArgs &, cudaStream_t);
void launch_y_70(const YArgs &, cudaStream_t);
void launch_y_72(const YArgs &, cudaStream_t);
void launch_y_75(const YArgs &, cudaStream_t);
void launch_y_80(const YArgs &, cudaStream_t);
void launch_y_81(const YArgs &, cudaStream_t);
void launch_y_84(const YArgs &, cudaStream_t);
void launch_y_90(const YArgs &, cudaStream_t);
void launch_y_96(const YArgs &, cudaStream_t);
void launch_y_98(const YArgs &, cudaStream_t);
void launch_y_100(const YArgs &, cudaStream_t);
void launch_y_105(const YArgs &, cudaStream_t);
void launch_y_108(const YArgs &, cudaStream_t);
void launch_y_112(const YArgs &, cudaStream_t);
void launch_y_120(const YArgs &, cudaStream_t);
void launch_y_125(const YArgs &, cudaStream_t);
void launch_y_126(const YArgs &, cudaStream_t);
void launch_y_128(const YArgs &, cudaStream_t);
void launch_y_135(const YArgs &, cudaStream_t);
void launch_y_140(const YArgs &, cudaStream_t);
void launch_y_144(const YArgs &, cudaStream_t);
void launch_y_147(const YArgs &, cudaStream_t);
void launch_y_150(const YArgs &, cudaStream_t);
void launch_y_160(const YArgs &, cudaStream_t);
void launch_y_162(const YArgs &, cudaStream_t);
void launch_y_168(const YArgs &, cudaStream_t);
void launch_y_175(const YArgs &, cudaStream_t);
void launch_y_180(const YArgs &, cudaStream_t);
void launch_y_189(const YArgs &, cudaStream_t);
void launch_y_192(const YArgs &, cudaStream_t);
void launch_y_196(const YArgs &, cudaStream_t);
void launch_y_200(const YArgs &, cudaStream_t);
void launch_y_210(const YArgs &, cudaStream_t);
void launch_y_216(const YArgs &, cudaStream_t);
void launch_y_224(const YArgs &, cudaStream_t);
void launch_y_225(const YArgs &, cudaStream_t);
void launch_y_240(const YArgs &, cudaStream_t);
void launch_y_243(const YArgs &, cudaStream_t);
void launch_y_245(const YArgs &, cudaStream_t);
void launch_y_250(const YArgs &, cudaStream_t);
void launch_y_252(const YArgs &, cudaStream_t);
void launch_y_256(const YArgs &, cudaStream_t);
void launch_y_270(const YArgs &, cudaStream_t);
void launch_y_280(const YArgs &, cudaStream_t);
void launch_y_288(const YArgs &, cudaStream_t);
void launch_y_294(const YArgs &, cudaStream_t);
void launch_y_300(const YArgs &, cudaStream_t);
void launch_y_315(const YArgs &, cudaStream_t);
void launch_y_320(const YArgs &, cudaStream_t);
void launch_y_324(const YArgs &, cudaStream_t);
void launch_y_336(const YArgs &, cudaStream_t);
void launch_y_343(const YArgs &, cudaStream_t);
void launch_y_350(const YArgs &, cudaStream_t);
void launch_y_360(const YArgs &, cudaStream_t);
void launch_y_375(const YArgs &, cudaStream_t);
void launch_y_378(const YArgs &, cudaStream_t);
void launch_y_384(const YArgs &, cudaStream_t);
void launch_y_392(const YArgs &, cudaStream_t);
void launch_y_400(const YArgs &, cudaStream_t);
void launch_y_405(const YArgs &, cudaStream_t);
void launch_y_420(const YArgs &, cudaStream_t);
void launch_y_432(const YArgs &, cudaStream_t);
void launch_y_441(const YArgs &, cudaStream_t);
void launch_y_448(const YArgs &, cudaStream_t);
void launch_y_450(const YArgs &, cudaStream_t);
void launch_y_480(const YArgs &, cudaStream_t);
void launch_y_486(const YArgs &, cudaStream_t);
void launch_y_490(const YArgs &, cudaStream_t);
void launch_y_500(const YArgs &, cudaStream_t);
void launch_y_504(const YArgs &, cudaStream_t);
void launch_y_512(const YArgs &, cudaStream_t);
void launch_y_525(const YArgs &, cudaStream_t);
void launch_y_540(const YArgs &, cudaStream_t);
void launch_y_560(const YArgs &, cudaStream_t);
void launch_y_567(const YArgs &, cudaStream_t);
void launch_y_576(const YArgs &, cudaStream_t);
void launch_y_588(const YArgs &, cudaStream_t);
void launch_y_600(const YArgs &, cudaStream_t);
void launch_y_630(const YArgs &, cudaStream_t);
void launch_y_640(const YArgs &, cudaStream_t);
void launch_y_648(const YArgs &, cudaStream_t);
void launch_y_672(const YArgs &, cudaStream_t);
void launch_y_675(const YArgs &, cudaStream_t);
void launch_y_686(const YArgs &, cudaStream_t);
void launch_y_700(const YArgs &, cudaStream_t);
void launch_y_720(const YArgs &, cudaStream_t);
void launch_y_729(const YArgs &, cudaStream_t);
void launch_y_735(const YArgs &, cudaStream_t);
void launch_y_750(const YArgs &, cudaStream_t);
void launch_y_756(const YArgs &, cudaStream_t);
void launch_y_768(const YArgs &, cudaStream_t);
void launch_y_784(const YArgs &, cudaStream_t);
void launch_y_800(const YArgs &, cudaStream_t);
void launch_y_810(const YArgs &, cudaStream_t);
void launch_y_840(const YArgs &, cudaStream_t);
void launch_y_864(const YArgs &, cudaStream_t);
void launch_y_882(const YArgs &, cudaStream_t);
void launch_y_896(const YArgs &, cudaStream_t);
void launch_y_900(const YArgs &, cudaStream_t);
void launch_y_945(const YArgs &, cudaStream_t);
void launch_y_960(const YArgs &, cudaStream_t);
void launch_y_972(const YArgs &, cudaStream_t);
void launch_y_980(const YArgs &, cudaStream_t);
void launch_y_1000(const YArgs &, cudaStream_t);
void launch_y_1008(const YArgs &, cudaStream_t);
void launch_y_1024(const YArgs &, cudaStream_t);
void launch_y_1050(const YArgs &, cudaStream_t);
void launch_y_1080(const YArgs &, cudaStream_t);
void launch_y_1120(const YArgs &, cudaStream_t);
void launch_y_1125(const YArgs &, cudaStream_t);
void launch_y_1134(const YArgs &, cudaStream_t);
void launch_y_1152(const YArgs &, cudaStream_t);
void launch_y_1176(const YArgs &, cudaStream_t);
void launch_y_1200(const YArgs &, cudaStream_t);
void launch_y_1215(const YArgs &, cudaStream_t);
void launch_y_1260(const YArgs &, cudaStream_t);
void launch_y_1280(const YArgs &, cudaStream_t);
void launch_y_1296(const YArgs &, cudaStream_t);
void launch_y_1344(const YArgs &, cudaStream_t);
void launch_y_1350(const YArgs &, cudaStream_t);
void launch_y_1372(const YArgs &, cudaStream_t);
void launch_y_1400(const YArgs &, cudaStream_t);
void launch_y_1440(const YArgs &, cudaStream_t);
void launch_y_1470(const YArgs &, cudaStream_t);
void launch_y_1500(const YArgs &, cudaStream_t);
void launch_y_1512(const YArgs &, cudaStream_t);
void launch_y_1536(const YArgs &, cudaStream_t);
void launch_y_1568(const YArgs &, cudaStream_t);
void launch_y_1575(const YArgs &, cudaStream_t);
void launch_y_1600(const YArgs &, cudaStream_t);
void launch_y_1620(const YArgs &, cudaStream_t);
void launch_y_1680(const YArgs &, cudaStream_t);
void launch_y_1728(const YArgs &, cudaStream_t);
void launch_y_1764(const YArgs &, cudaStream_t);
void launch_y_1792(const YArgs &, cudaStream_t);
void launch_y_1800(const YArgs &, cudaStream_t);
void launch_y_1890(const YArgs &, cudaStream_t);
void launch_y_1920(const YArgs &, cudaStream_t);
void launch_y_1960(const YArgs &, cudaStream_t);
void launch_y_2016(const YArgs &, cudaStream_t);
void launch_y_2025(const YArgs &, cudaStream_t);
void launch_y_2048(const YArgs &, cudaStream_t);
void launch_y_2100(const YArgs &, cudaStream_t);
void launch_y_2160(const YArgs &, cudaStream_t);
void launch_y_2240(const YArgs &, cudaStream_t);
void launch_y_2250(const YArgs &, cudaStream_t);
void launch_y_2304(const YArgs &, cudaStream_t);
void launch_y_2352(const YArgs &, cudaStream_t);
void launch_y_2400(const YArgs &, cudaStream_t);
void launch_y_2520(const YArgs &, cudaStream_t);
void launch_y_2560(const YArgs &, cudaStream_t);
void launch_y_2688(const YArgs &, cudaStream_t);
void launch_y_2700(const YArgs &, cudaStream_t);
void launch_y_2744(const YArgs &, cudaStream_t);
void launch_y_2880(const YArgs &, cudaStream_t);
void launch_y_2940(const YArgs &, cudaStream_t);
void launch_y_3072(const YArgs &, cudaStream_t);
void launch_y_3136(const YArgs &, cudaStream_t);
void launch_y_3150(const YArgs &, cudaStream_t);
static const LinesPlan kLinesPlans[] = {
    {1, 1, 1, 1, 16, LinesCfg<Rad<1, 1, 1>, 16>::THREADS, LinesCfg<Rad<1, 1, 1>, 16>::SMEM_BYTES, launch_lines_1},
    {2, 2, 1, 1, 16, LinesCfg<Rad<2, 1, 1>, 16>::THREADS, LinesCfg<Rad<2, 1, 1>, 16>::SMEM_BYTES, launch_lines_2},
    {3, 3, 1, 1, 16, LinesCfg<Rad<3, 1, 1>, 16>::THREADS, LinesCfg<Rad<3, 1, 1>, 16>::SMEM_BYTES, launch_lines_3},
    {4, 2, 2, 1, 16, LinesCfg<Rad<2, 2, 1>, 16>::THREADS, LinesCfg<Rad<2, 2, 1>, 16>::SMEM_BYTES, launch_lines_4},
    {5, 5, 1, 1, 16, LinesCfg<Rad<5, 1, 1>, 16>::THREADS, LinesCfg<Rad<5, 1, 1>, 16>::SMEM_BYTES, launch_lines_5},
    {6, 3, 2, 1, 16, LinesCfg<Rad<3, 2, 1>, 16>::THREADS, LinesCfg<Rad<3, 2, 1>, 16>::SMEM_BYTES, launch_lines_6},
    {7, 7, 1, 1, 16, LinesCfg<Rad<7, 1, 1>, 16>::THREADS, LinesCfg<Rad<7, 1, 1>, 16>::SMEM_BYTES, launch_lines_7},
    {8, 4, 2, 1, 16, LinesCfg<Rad<4, 2, 1>, 16>::THREADS, LinesCfg<Rad<4, 2, 1>, 16>::SMEM_BYTES, launch_lines_8},
    {9, 3, 3, 1, 16, LinesCfg<Rad<3, 3, 1>, 16>::THREADS, LinesCfg<Rad<3, 3, 1>, 16>::SMEM_BYTES, launch_lines_9},
    {10, 5, 2, 1, 16, LinesCfg<Rad<5, 2, 1>, 16>::THREADS, LinesCfg<Rad<5, 2, 1>, 16>::SMEM_BYTES, launch_lines_10},
    {12, 4, 3, 1, 16, LinesCfg<Rad<4, 3, 1>, 16>::THREADS, LinesCfg<Rad<4, 3, 1>, 16>::SMEM_BYTES, launch_lines_12},
    {14, 7, 2, 1, 16, LinesCfg<Rad<7, 2, 1>, 16>::THREADS, LinesCfg<Rad<7, 2, 1>, 16>::SMEM_BYTES, launch_lines_14},
    {15, 5, 3, 1, 16, LinesCfg<Rad<5, 3, 1>, 16>::THREADS, LinesCfg<Rad<5, 3, 1>, 16>::SMEM_BYTES, launch_lines_15},
    {16, 4, 4, 1, 16, LinesCfg<Rad<4, 4, 1>, 16>::THREADS, LinesCfg<Rad<4, 4, 1>, 16>::SMEM_BYTES, launch_lines_16},
    {18, 6, 3, 1, 16, LinesCfg<Rad<6, 3, 1>, 16>::THREADS, LinesCfg<Rad<6, 3, 1>, 16>::SMEM_BYTES, launch_lines_18},
    {20, 5, 4, 1, 16, LinesCfg<Rad<5, 4, 1>, 16>::THREADS, LinesCfg<Rad<5, 4, 1>, 16>::SMEM_BYTES, launch_lines_20},
    {21, 7, 3, 1, 16, LinesCfg<Rad<7, 3, 1>, 16>::THREADS, LinesCfg<Rad<7, 3, 1>, 16>::SMEM_BYTES, launch_lines_21},
    {24, 6, 4, 1, 16, LinesCfg<Rad<6, 4, 1>, 16>::THREADS, LinesCfg<Rad<6, 4, 1>, 16>::SMEM_BYTES, launch_lines_24},
    {25, 5, 5, 1, 16, LinesCfg<Rad<5, 5, 1>, 16>::THREADS, LinesCfg<Rad<5, 5, 1>, 16>::SMEM_BYTES, launch_lines_25},
    {27, 9, 3, 1, 16, LinesCfg<Rad<9, 3, 1>, 16>::THREADS, LinesCfg<Rad<9, 3, 1>, 16>::SMEM_BYTES, launch_lines_27},
    {28, 7, 4, 1, 16, LinesCfg<Rad<7, 4, 1>, 16>::THREADS, LinesCfg<Rad<7, 4, 1>, 16>::SMEM_BYTES, launch_lines_28},
    {30, 6, 5, 1, 16, LinesCfg<Rad<6, 5, 1>, 16>::THREADS, LinesCfg<Rad<6, 5, 1>, 16>::SMEM_BYTES, launch_lines_30},
    {32, 8, 4, 1, 16, LinesCfg<Rad<8, 4, 1>, 16>::THREADS, LinesCfg<Rad<8, 4, 1>, 16>::SMEM_BYTES, launch_lines_32},
    {35, 7, 5, 1, 16, LinesCfg<Rad<7, 5, 1>, 16>::THREADS, LinesCfg<Rad<7, 5, 1>, 16>::SMEM_BYTES, launch_lines_35},
    {36, 6, 6, 1, 16, LinesCfg<Rad<6, 6, 1>, 16>::THREADS, LinesCfg<Rad<6, 6, 1>, 16>::SMEM_BYTES, launch_lines_36},
    {40, 8, 5, 1, 16, LinesCfg<Rad<8, 5, 1>, 16>::THREADS, LinesCfg<Rad<8, 5, 1>, 16>::SMEM_BYTES, launch_lines_40},
    {42, 7, 6, 1, 16, LinesCfg<Rad<7, 6, 1>, 16>::THREADS, LinesCfg<Rad<7, 6, 1>, 16>::SMEM_BYTES, launch_lines_42},
    {45, 9, 5, 1, 16, LinesCfg<Rad<9, 5, 1>, 16>::THREADS, LinesCfg<Rad<9, 5, 1>, 16>::SMEM_BYTES, launch_lines_45},
    {48, 8, 6, 1, 16, LinesCfg<Rad<8, 6, 1>, 16>::THREADS, LinesCfg<Rad<8, 6, 1>, 16>::SMEM_BYTES, launch_lines_48},
    {49, 7, 7, 1, 16, LinesCfg<Rad<7, 7, 1>, 16>::THREADS, LinesCfg<Rad<7, 7, 1>, 16>::SMEM_BYTES, launch_lines_49},
    {50, 10, 5, 1, 16, LinesCfg<Rad<10, 5, 1>, 16>::THREADS, LinesCfg<Rad<10, 5, 1>, 16>::SMEM_BYTES, launch_lines_50},
    {54, 9, 6, 1, 16, LinesCfg<Rad<9, 6, 1>, 16>::THREADS, LinesCfg<Rad<9, 6, 1>, 16>::SMEM_BYTES, launch_lines_54},
    {56, 8, 7, 1, 16, LinesCfg<Rad<8, 7, 1>, 16>::THREADS, LinesCfg<Rad<8, 7, 1>, 16>::SMEM_BYTES, launch_lines_56},
    {60, 10, 6, 1, 16, LinesCfg<Rad<10, 6, 1>, 16>::THREADS, LinesCfg<Rad<10, 6, 1>, 16>::SMEM_BYTES, launch_lines_60},
    {63, 9, 7, 1, 16, LinesCfg<Rad<9, 7, 1>, 16>::THREADS, LinesCfg<Rad<9, 7, 1>, 16>::SMEM_BYTES, launch_lines_63},
    {64, 8, 8, 1, 16, LinesCfg<Rad<8, 8, 1>, 16>::THREADS, LinesCfg<Rad<8, 8, 1>, 16>::SMEM_BYTES, launch_lines_64},
    {70, 10, 7, 1, 16, LinesCfg<Rad<10, 7, 1>, 16>::THREADS, LinesCfg<Rad<10, 7, 1>, 16>::SMEM_BYTES, launch_lines_70},
    {72, 9, 8, 1, 16, LinesCfg<Rad<9, 8, 1>, 16>::THREADS, LinesCfg<Rad<9, 8, 1>, 16>::SMEM_BYTES, launch_lines_72},
    {75, 15, 5, 1, 16, LinesCfg<Rad<15, 5, 1>, 16>::THREADS, LinesCfg<Rad<15, 5, 1>, 16>::SMEM_BYTES, launch_lines_75},
    {80, 10, 8, 1, 16, LinesCfg<Rad<10, 8, 1>, 16>::THREADS, LinesCfg<Rad<10, 8, 1>, 16>::SMEM_BYTES, launch_lines_80},
    {81, 9, 9, 1, 16, LinesCfg<Rad<9, 9, 1>, 16>::THREADS, LinesCfg<Rad<9, 9, 1>, 16>::SMEM_BYTES, launch_lines_81},
    {84, 12, 7, 1, 16, LinesCfg<Rad<12, 7, 1>, 16>::THREADS, LinesCfg<Rad<12, 7, 1>, 16>::SMEM_BYTES, launch_lines_84},
    {90, 10, 9, 1, 16, LinesCfg<Rad<10, 9, 1>, 16>::THREADS, LinesCfg<Rad<10, 9, 1>, 16>::SMEM_BYTES, launch_lines_90},
    {96, 12, 8, 1, 16, LinesCfg<Rad<12, 8, 1>, 16>::THREADS, LinesCfg<Rad<12, 8, 1>, 16>::SMEM_BYTES, launch_lines_96},
    {98, 14, 7, 1, 16, LinesCfg<Rad<14, 7, 1>, 16>::THREADS, LinesCfg<Rad<14, 7, 1>, 16>::SMEM_BYTES, launch_lines_98},
    {100, 10, 10, 1, 16, LinesCfg<Rad<10, 10, 1>, 16>::THREADS, LinesCfg<Rad<10, 10, 1>, 16>::SMEM_BYTES, launch_lines_100},
    {105, 15, 7, 1, 16, LinesCfg<Rad<15, 7, 1>, 16>::THREADS, LinesCfg<Rad<15, 7, 1>, 16>::SMEM_BYTES, launch_lines_105},
    {108, 12, 9, 1, 16, LinesCfg<Rad<12, 9, 1>, 16>::THREADS, LinesCfg<Rad<12, 9, 1>, 16>::SMEM_BYTES, launch_lines_108},
    {112, 14, 8, 1, 16, LinesCfg<Rad<14, 8, 1>, 16>::THREADS, LinesCfg<Rad<14, 8, 1>, 16>::SMEM_BYTES, launch_lines_112},
    {120, 12, 10, 1, 16, LinesCfg<Rad<12, 10, 1>, 16>::THREADS, LinesCfg<Rad<12, 10, 1>, 16>::SMEM_BYTES, launch_lines_120},
    {125, 5, 5, 5, 16, LinesCfg<Rad<5, 5, 5>, 16>::THREADS, LinesCfg<Rad<5, 5, 5>, 16>::SMEM_BYTES, launch_lines_125},
    {126, 14, 9, 1, 16, LinesCfg<Rad<14, 9, 1>, 16>::THREADS, LinesCfg<Rad<14, 9, 1>, 16>::SMEM_BYTES, launch_lines_126},
    {128, 16, 8, 1, 16, LinesCfg<Rad<16, 8, 1>, 16>::THREADS, LinesCfg<Rad<16, 8, 1>, 16>::SMEM_BYTES, launch_lines_128},
    {135, 15, 9, 1, 16, LinesCfg<Rad<15, 9, 1>, 16>::THREADS, LinesCfg<Rad<15, 9, 1>, 16>::SMEM_BYTES, launch_lines_135},
    {140, 14, 10, 1, 16, LinesCfg<Rad<14, 10, 1>, 16>::THREADS, LinesCfg<Rad<14, 10, 1>, 16>::SMEM_BYTES, launch_lines_140},
    {144, 12, 12, 1, 16, LinesCfg<Rad<12, 12, 1>, 16>::THREADS, LinesCfg<Rad<12, 12, 1>, 16>::SMEM_BYTES, launch_lines_144},
    {147, 7, 3, 7, 16, LinesCfg<Rad<7, 3, 7>, 16>::THREADS, LinesCfg<Rad<7, 3, 7>, 16>::SMEM_BYTES, launch_lines_147},
    {150, 15, 10, 1, 16, LinesCfg<Rad<15, 10, 1>, 16>::THREADS, LinesCfg<Rad<15, 10, 1>, 16>::SMEM_BYTES, launch_lines_150},
    {160, 16, 10, 1, 16, LinesCfg<Rad<16, 10, 1>, 16>::THREADS, LinesCfg<Rad<16, 10, 1>, 16>::SMEM_BYTES, launch_lines_160},
    {162, 9, 3, 6, 16, LinesCfg<Rad<9, 3, 6>, 16>::THREADS, LinesCfg<Rad<9, 3, 6>, 16>::SMEM_BYTES, launch_lines_162},
    {168, 14, 12, 1, 16, LinesCfg<Rad<14, 12, 1>, 16>::THREADS, LinesCfg<Rad<14, 12, 1>, 16>::SMEM_BYTES, launch_lines_168},
    {175, 7, 5, 5, 16, LinesCfg<Rad<7, 5, 5>, 16>::THREADS, LinesCfg<Rad<7, 5, 5>, 16>::SMEM_BYTES, launch_lines_175},
    {180, 15, 12, 1, 16, LinesCfg<Rad<15, 12, 1>, 16>::THREADS, LinesCfg<Rad<15, 12, 1>, 16>::SMEM_BYTES, launch_lines_180},
    {189, 9, 3, 7, 16, LinesCfg<Rad<9, 3, 7>, 16>::THREADS, LinesCfg<Rad<9, 3, 7>, 16>::SMEM_BYTES, launch_lines_189},
    {192, 16, 12, 1, 16, LinesCfg<Rad<16, 12, 1>, 16>::THREADS, LinesCfg<Rad<16, 12, 1>, 16>::SMEM_BYTES, launch_lines_192},
    {196, 14, 14, 1, 16, LinesCfg<Rad<14, 14, 1>, 16>::THREADS, LinesCfg<Rad<14, 14, 1>, 16>::SMEM_BYTES, launch_lines_196},
    {200, 8, 5, 5, 16, LinesCfg<Rad<8, 5, 5>, 16>::THREADS, LinesCfg<Rad<8, 5, 5>, 16>::SMEM_BYTES, launch_lines_200},
    {210, 15, 14, 1, 16, LinesCfg<Rad<15, 14, 1>, 16>::THREADS, LinesCfg<Rad<15, 14, 1>, 16>::SMEM_BYTES, launch_lines_210},
    {216, 6, 6, 6, 16, LinesCfg<Rad<6, 6, 6>, 16>::THREADS, LinesCfg<Rad<6, 6, 6>, 16>::SMEM_BYTES, launch_lines_216},
    {224, 16, 14, 1, 16, LinesCfg<Rad<16, 14, 1>, 16>::THREADS, LinesCfg<Rad<16, 14, 1>, 16>::SMEM_BYTES, launch_lines_224},
    {225, 15, 15, 1, 16, LinesCfg<Rad<15, 15, 1>, 16>::THREADS, LinesCfg<Rad<15, 15, 1>, 16>::SMEM_BYTES, launch_lines_225},
    {240, 16, 15, 1, 16, LinesCfg<Rad<16, 15, 1>, 16>::THREADS, LinesCfg<Rad<16, 15, 1>, 16>::SMEM_BYTES, launch_lines_240},
    {243, 9, 3, 9, 8, LinesCfg<Rad<9, 3, 9>, 8>::THREADS, LinesCfg<Rad<9, 3, 9>, 8>::SMEM_BYTES, launch_lines_243},
    {245, 7, 5, 7, 16, LinesCfg<Rad<7, 5, 7>, 16>::THREADS, LinesCfg<Rad<7, 5, 7>, 16>::SMEM_BYTES, launch_lines_245},
    {250, 10, 5, 5, 16, LinesCfg<Rad<10, 5, 5>, 16>::THREADS, LinesCfg<Rad<10, 5, 5>, 16>::SMEM_BYTES, launch_lines_250},
    {252, 7, 6, 6, 16, LinesCfg<Rad<7, 6, 6>, 16>::THREADS, LinesCfg<Rad<7, 6, 6>, 16>::SMEM_BYTES, launch_lines_252},
    {256, 16, 16, 1, 16, LinesCfg<Rad<16, 16, 1>, 16>::THREADS, LinesCfg<Rad<16, 16, 1>, 16>::SMEM_BYTES, launch_lines_256},
    {270, 9, 5, 6, 16, LinesCfg<Rad<9, 5, 6>, 16>::THREADS, LinesCfg<Rad<9, 5, 6>, 16>::SMEM_BYTES, launch_lines_270},
    {280, 8, 5, 7, 16, LinesCfg<Rad<8, 5, 7>, 16>::THREADS, LinesCfg<Rad<8, 5, 7>, 16>::SMEM_BYTES, launch_lines_280},
    {288, 8, 6, 6, 16, LinesCfg<Rad<8, 6, 6>, 16>::THREADS, LinesCfg<Rad<8, 6, 6>, 16>::SMEM_BYTES, launch_lines_288},
    {294, 7, 6, 7, 16, LinesCfg<Rad<7, 6, 7>, 16>::THREADS, LinesCfg<Rad<7, 6, 7>, 16>::SMEM_BYTES, launch_lines_294},
    {300, 10, 5, 6, 16, LinesCfg<Rad<10, 5, 6>, 16>::THREADS, LinesCfg<Rad<10, 5, 6>, 16>::SMEM_BYTES, launch_lines_300},
    {315, 9, 5, 7, 16, LinesCfg<Rad<9, 5, 7>, 16>::THREADS, LinesCfg<Rad<9, 5, 7>, 16>::SMEM_BYTES, launch_lines_315},
    {320, 8, 5, 8, 16, LinesCfg<Rad<8, 5, 8>, 16>::THREADS, LinesCfg<Rad<8, 5, 8>, 16>::SMEM_BYTES, launch_lines_320},
    {324, 9, 6, 6, 16, LinesCfg<Rad<9, 6, 6>, 16>::THREADS, LinesCfg<Rad<9, 6, 6>, 16>::SMEM_BYTES, launch_lines_324},
    {336, 8, 6, 7, 16, LinesCfg<Rad<8, 6, 7>, 16>::THREADS, LinesCfg<Rad<8, 6, 7>, 16>::SMEM_BYTES, launch_lines_336},
    {343, 7, 7, 7, 16, LinesCfg<Rad<7, 7, 7>, 16>::THREADS, LinesCfg<Rad<7, 7, 7>, 16>::SMEM_BYTES, launch_lines_343},
    {350, 10, 5, 7, 8, LinesCfg<Rad<10, 5, 7>, 8>::THREADS, LinesCfg<Rad<10, 5, 7>, 8>::SMEM_BYTES, launch_lines_350},
    {360, 10, 6, 6, 16, LinesCfg<Rad<10, 6, 6>, 16>::THREADS, LinesCfg<Rad<10, 6, 6>, 16>::SMEM_BYTES, launch_lines_360},
    {375, 15, 5, 5, 8, LinesCfg<Rad<15, 5, 5>, 8>::THREADS, LinesCfg<Rad<15, 5, 5>, 8>::SMEM_BYTES, launch_lines_375},
    {378, 9, 6, 7, 16, LinesCfg<Rad<9, 6, 7>, 16>::THREADS, LinesCfg<Rad<9, 6, 7>, 16>::SMEM_BYTES, launch_lines_378},
    {384, 8, 6, 8, 16, LinesCfg<Rad<8, 6, 8>, 16>::THREADS, LinesCfg<Rad<8, 6, 8>, 16>::SMEM_BYTES, launch_lines_384},
    {392, 8, 7, 7, 16, LinesCfg<Rad<8, 7, 7>, 16>::THREADS, LinesCfg<Rad<8, 7, 7>, 16>::SMEM_BYTES, launch_lines_392},
    {400, 10, 5, 8, 8, LinesCfg<Rad<10, 5, 8>, 8>::THREADS, LinesCfg<Rad<10, 5, 8>, 8>::SMEM_BYTES, launch_lines_400},
    {405, 9, 5, 9, 8, LinesCfg<Rad<9, 5, 9>, 8>::THREADS, LinesCfg<Rad<9, 5, 9>, 8>::SMEM_BYTES, launch_lines_405},
    {420, 10, 6, 7, 8, LinesCfg<Rad<10, 6, 7>, 8>::THREADS, LinesCfg<Rad<10, 6, 7>, 8>::SMEM_BYTES, launch_lines_420},
    {432, 9, 6, 8, 8, LinesCfg<Rad<9, 6, 8>, 8>::THREADS, LinesCfg<Rad<9, 6, 8>, 8>::SMEM_BYTES, launch_lines_432},
    {441, 9, 7, 7, 16, LinesCfg<Rad<9, 7, 7>, 16>::THREADS, LinesCfg<Rad<9, 7, 7>, 16>::SMEM_BYTES, launch_lines_441},
    {448, 8, 7, 8, 16, LinesCfg<Rad<8, 7, 8>, 16>::THREADS, LinesCfg<Rad<8, 7, 8>, 16>::SMEM_BYTES, launch_lines_448},
    {450, 10, 5, 9, 8, LinesCfg<Rad<10, 5, 9>, 8>::THREADS, LinesCfg<Rad<10, 5, 9>, 8>::SMEM_BYTES, launch_lines_450},
    {480, 10, 6, 8, 8, LinesCfg<Rad<10, 6, 8>, 8>::THREADS, LinesCfg<Rad<10, 6, 8>, 8>::SMEM_BYTES, launch_lines_480},
    {486, 9, 6, 9, 8, LinesCfg<Rad<9, 6, 9>, 8>::THREADS, LinesCfg<Rad<9, 6, 9>, 8>::SMEM_BYTES, launch_lines_486},
    {490, 10, 7, 7, 8, LinesCfg<Rad<10, 7, 7>, 8>::THREADS, LinesCfg<Rad<10, 7, 7>, 8>::SMEM_BYTES, launch_lines_490},
    {500, 10, 5, 10, 8, LinesCfg<Rad<10, 5, 10>, 8>::THREADS, LinesCfg<Rad<10, 5, 10>, 8>::SMEM_BYTES, launch_lines_500},
    {504, 9, 7, 8, 8, LinesCfg<Rad<9, 7, 8>, 8>::THREADS, LinesCfg<Rad<9, 7, 8>, 8>::SMEM_BYTES, launch_lines_504},
    {512, 8, 8, 8, 16, LinesCfg<Rad<8, 8, 8>, 16>::THREADS, LinesCfg<Rad<8, 8, 8>, 16>::SMEM_BYTES, launch_lines_512},
    {525, 15, 5, 7, 8, LinesCfg<Rad<15, 5, 7>, 8>::THREADS, LinesCfg<Rad<15, 5, 7>, 8>::SMEM_BYTES, launch_lines_525},
    {540, 10, 6, 9, 8, LinesCfg<Rad<10, 6, 9>, 8>::THREADS, LinesCfg<Rad<10, 6, 9>, 8>::SMEM_BYTES, launch_lines_540},
    {560, 10, 7, 8, 8, LinesCfg<Rad<10, 7, 8>, 8>::THREADS, LinesCfg<Rad<10, 7, 8>, 8>::SMEM_BYTES, launch_lines_560},
    {567, 9, 7, 9, 8, LinesCfg<Rad<9, 7, 9>, 8>::THREADS, LinesCfg<Rad<9, 7, 9>, 8>::SMEM_BYTES, launch_lines_567},
    {576, 9, 8, 8, 8, LinesCfg<Rad<9, 8, 8>, 8>::THREADS, LinesCfg<Rad<9, 8, 8>, 8>::SMEM_BYTES, launch_lines_576},
    {588, 12, 7, 7, 8, LinesCfg<Rad<12, 7, 7>, 8>::THREADS, LinesCfg<Rad<12, 7, 7>, 8>::SMEM_BYTES, launch_lines_588},
    {600, 10, 6, 10, 8, LinesCfg<Rad<10, 6, 10>, 8>::THREADS, LinesCfg<Rad<10, 6, 10>, 8>::SMEM_BYTES, launch_lines_600},
    {630, 10, 7, 9, 8, LinesCfg<Rad<10, 7, 9>, 8>::THREADS, LinesCfg<Rad<10, 7, 9>, 8>::SMEM_BYTES, launch_lines_630},
    {640, 10, 8, 8, 8, LinesCfg<Rad<10, 8, 8>, 8>::THREADS, LinesCfg<Rad<10, 8, 8>, 8>::SMEM_BYTES, launch_lines_640},
    {648, 9, 8, 9, 8, LinesCfg<Rad<9, 8, 9>, 8>::THREADS, LinesCfg<Rad<9, 8, 9>, 8>::SMEM_BYTES, launch_lines_648},
    {672, 12, 7, 8, 8, LinesCfg<Rad<12, 7, 8>, 8>::THREADS, LinesCfg<Rad<12, 7, 8>, 8>::SMEM_BYTES, launch_lines_672},
    {675, 15, 5, 9, 4, LinesCfg<Rad<15, 5, 9>, 4>::THREADS, LinesCfg<Rad<15, 5, 9>, 4>::SMEM_BYTES, launch_lines_675},
    {686, 14, 7, 7, 8, LinesCfg<Rad<14, 7, 7>, 8>::THREADS, LinesCfg<Rad<14, 7, 7>, 8>::SMEM_BYTES, launch_lines_686},
    {700, 10, 7, 10, 8, LinesCfg<Rad<10, 7, 10>, 8>::THREADS, LinesCfg<Rad<10, 7, 10>, 8>::SMEM_BYTES, launch_lines_700},
    {720, 10, 8, 9, 8, LinesCfg<Rad<10, 8, 9>, 8>::THREADS, LinesCfg<Rad<10, 8, 9>, 8>::SMEM_BYTES, launch_lines_720},
    {729, 9, 9, 9, 8, LinesCfg<Rad<9, 9, 9>, 8>::THREADS, LinesCfg<Rad<9, 9, 9>, 8>::SMEM_BYTES, launch_lines_729},
    {735, 15, 7, 7, 8, LinesCfg<Rad<15, 7, 7>, 8>::THREADS, LinesCfg<Rad<15, 7, 7>, 8>::SMEM_BYTES, launch_lines_735},
    {750, 15, 5, 10, 4, LinesCfg<Rad<15, 5, 10>, 4>::THREADS, LinesCfg<Rad<15, 5, 10>, 4>::SMEM_BYTES, launch_lines_750},
    {756, 12, 7, 9, 8, LinesCfg<Rad<12, 7, 9>, 8>::THREADS, LinesCfg<Rad<12, 7, 9>, 8>::SMEM_BYTES, launch_lines_756},
    {768, 12, 8, 8, 8, LinesCfg<Rad<12, 8, 8>, 8>::THREADS, LinesCfg<Rad<12, 8, 8>, 8>::SMEM_BYTES, launch_lines_768},
    {784, 14, 7, 8, 8, LinesCfg<Rad<14, 7, 8>, 8>::THREADS, LinesCfg<Rad<14, 7, 8>, 8>::SMEM_BYTES, launch_lines_784},
    {800, 10, 8, 10, 8, LinesCfg<Rad<10, 8, 10>, 8>::THREADS, LinesCfg<Rad<10, 8, 10>, 8>::SMEM_BYTES, launch_lines_800},
    {810, 10, 9, 9, 8, LinesCfg<Rad<10, 9, 9>, 8>::THREADS, LinesCfg<Rad<10, 9, 9>, 8>::SMEM_BYTES, launch_lines_810},
    {840, 12, 7, 10, 8, LinesCfg<Rad<12, 7, 10>, 8>::THREADS, LinesCfg<Rad<12, 7, 10>, 8>::SMEM_BYTES, launch_lines_840},
    {864, 12, 8, 9, 8, LinesCfg<Rad<12, 8, 9>, 8>::THREADS, LinesCfg<Rad<12, 8, 9>, 8>::SMEM_BYTES, launch_lines_864},
    {882, 14, 7, 9, 8, LinesCfg<Rad<14, 7, 9>, 8>::THREADS, LinesCfg<Rad<14, 7, 9>, 8>::SMEM_BYTES, launch_lines_882},
    {896, 14, 8, 8, 8, LinesCfg<Rad<14, 8, 8>, 8>::THREADS, LinesCfg<Rad<14, 8, 8>, 8>::SMEM_BYTES, launch_lines_896},
    {900, 10, 9, 10, 8, LinesCfg<Rad<10, 9, 10>, 8>::THREADS, LinesCfg<Rad<10, 9, 10>, 8>::SMEM_BYTES, launch_lines_900},
    {945, 15, 7, 9, 4, LinesCfg<Rad<15, 7, 9>, 4>::THREADS, LinesCfg<Rad<15, 7, 9>, 4>::SMEM_BYTES, launch_lines_945},
    {960, 12, 8, 10, 8, LinesCfg<Rad<12, 8, 10>, 8>::THREADS, LinesCfg<Rad<12, 8, 10>, 8>::SMEM_BYTES, launch_lines_960},
    {972, 12, 9, 9, 8, LinesCfg<Rad<12, 9, 9>, 8>::THREADS, LinesCfg<Rad<12, 9, 9>, 8>::SMEM_BYTES, launch_lines_972},
    {980, 14, 7, 10, 4, LinesCfg<Rad<14, 7, 10>, 4>::THREADS, LinesCfg<Rad<14, 7, 10>, 4>::SMEM_BYTES, launch_lines_980},
    {1000, 10, 10, 10, 8, LinesCfg<Rad<10, 10, 10>, 8>::THREADS, LinesCfg<Rad<10, 10, 10>, 8>::SMEM_BYTES, launch_lines_1000},
    {1008, 14, 8, 9, 8, LinesCfg<Rad<14, 8, 9>, 8>::THREADS, LinesCfg<Rad<14, 8, 9>, 8>::SMEM_BYTES, launch_lines_1008},
    {1024, 16, 8, 8, 8, LinesCfg<Rad<16, 8, 8>, 8>::THREADS, LinesCfg<Rad<16, 8, 8>, 8>::SMEM_BYTES, launch_lines_1024},
    {1050, 15, 7, 10, 4, LinesCfg<Rad<15, 7, 10>, 4>::THREADS, LinesCfg<Rad<15, 7, 10>, 4>::SMEM_BYTES, launch_lines_1050},
    {1080, 12, 9, 10, 8, LinesCfg<Rad<12, 9, 10>, 8>::THREADS, LinesCfg<Rad<12, 9, 10>, 8>::SMEM_BYTES, launch_lines_1080},
    {1120, 14, 8, 10, 4, LinesCfg<Rad<14, 8, 10>, 4>::THREADS, LinesCfg<Rad<14, 8, 10>, 4>::SMEM_BYTES, launch_lines_1120},
    {1125, 15, 5, 15, 4, LinesCfg<Rad<15, 5, 15>, 4>::THREADS, LinesCfg<Rad<15, 5, 15>, 4>::SMEM_BYTES, launch_lines_1125},
    {1134, 14, 9, 9, 8, LinesCfg<Rad<14, 9, 9>, 8>::THREADS, LinesCfg<Rad<14, 9, 9>, 8>::SMEM_BYTES, launch_lines_1134},
    {1152, 12, 8, 12, 4, LinesCfg<Rad<12, 8, 12>, 4>::THREADS, LinesCfg<Rad<12, 8, 12>, 4>::SMEM_BYTES, launch_lines_1152},
    {1176, 14, 7, 12, 4, LinesCfg<Rad<14, 7, 12>, 4>::THREADS, LinesCfg<Rad<14, 7, 12>, 4>::SMEM_BYTES, launch_lines_1176},
    {1200, 12, 10, 10, 8, LinesCfg<Rad<12, 10, 10>, 8>::THREADS, LinesCfg<Rad<12, 10, 10>, 8>::SMEM_BYTES, launch_lines_1200},
    {1215, 15, 9, 9, 4, LinesCfg<Rad<15, 9, 9>, 4>::THREADS, LinesCfg<Rad<15, 9, 9>, 4>::SMEM_BYTES, launch_lines_1215},
    {1260, 14, 9, 10, 4, LinesCfg<Rad<14, 9, 10>, 4>::THREADS, LinesCfg<Rad<14, 9, 10>, 4>::SMEM_BYTES, launch_lines_1260},
    {1280, 16, 8, 10, 4, LinesCfg<Rad<16, 8, 10>, 4>::THREADS, LinesCfg<Rad<16, 8, 10>, 4>::SMEM_BYTES, launch_lines_1280},
    {1296, 12, 9, 12, 4, LinesCfg<Rad<12, 9, 12>, 4>::THREADS, LinesCfg<Rad<12, 9, 12>, 4>::SMEM_BYTES, launch_lines_1296},
    {1344, 14, 8, 12, 4, LinesCfg<Rad<14, 8, 12>, 4>::THREADS, LinesCfg<Rad<14, 8, 12>, 4>::SMEM_BYTES, launch_lines_1344},
    {1350, 15, 9, 10, 4, LinesCfg<Rad<15, 9, 10>, 4>::THREADS, LinesCfg<Rad<15, 9, 10>, 4>::SMEM_BYTES, launch_lines_1350},
    {1372, 14, 7, 14, 4, LinesCfg<Rad<14, 7, 14>, 4>::THREADS, LinesCfg<Rad<14, 7, 14>, 4>::SMEM_BYTES, launch_lines_1372},
    {1400, 14, 10, 10, 4, LinesCfg<Rad<14, 10, 10>, 4>::THREADS, LinesCfg<Rad<14, 10, 10>, 4>::SMEM_BYTES, launch_lines_1400},
    {1440, 12, 10, 12, 4, LinesCfg<Rad<12, 10, 12>, 4>::THREADS, LinesCfg<Rad<12, 10, 12>, 4>::SMEM_BYTES, launch_lines_1440},
    {1470, 15, 7, 14, 4, LinesCfg<Rad<15, 7, 14>, 4>::THREADS, LinesCfg<Rad<15, 7, 14>, 4>::SMEM_BYTES, launch_lines_1470},
    {1500, 15, 10, 10, 4, LinesCfg<Rad<15, 10, 10>, 4>::THREADS, LinesCfg<Rad<15, 10, 10>, 4>::SMEM_BYTES, launch_lines_1500},
    {1512, 14, 9, 12, 4, LinesCfg<Rad<14, 9, 12>, 4>::THREADS, LinesCfg<Rad<14, 9, 12>, 4>::SMEM_BYTES, launch_lines_1512},
    {1536, 16, 8, 12, 4, LinesCfg<Rad<16, 8, 12>, 4>::THREADS, LinesCfg<Rad<16, 8, 12>, 4>::SMEM_BYTES, launch_lines_1536},
    {1568, 14, 8, 14, 4, LinesCfg<Rad<14, 8, 14>, 4>::THREADS, LinesCfg<Rad<14, 8, 14>, 4>::SMEM_BYTES, launch_lines_1568},
    {1575, 15, 7, 15, 4, LinesCfg<Rad<15, 7, 15>, 4>::THREADS, LinesCfg<Rad<15, 7, 15>, 4>::SMEM_BYTES, launch_lines_1575},
    {1600, 16, 10, 10, 4, LinesCfg<Rad<16, 10, 10>, 4>::THREADS, LinesCfg<Rad<16, 10, 10>, 4>::SMEM_BYTES, launch_lines_1600},
    {1620, 15, 9, 12, 4, LinesCfg<Rad<15, 9, 12>, 4>::THREADS, LinesCfg<Rad<15, 9, 12>, 4>::SMEM_BYTES, launch_lines_1620},
    {1680, 14, 10, 12, 4, LinesCfg<Rad<14, 10, 12>, 4>::THREADS, LinesCfg<Rad<14, 10, 12>, 4>::SMEM_BYTES, launch_lines_1680},
    {1728, 12, 12, 12, 4, LinesCfg<Rad<12, 12, 12>, 4>::THREADS, LinesCfg<Rad<12, 12, 12>, 4>::SMEM_BYTES, launch_lines_1728},
    {1764, 14, 9, 14, 4, LinesCfg<Rad<14, 9, 14>, 4>::THREADS, LinesCfg<Rad<14, 9, 14>, 4>::SMEM_BYTES, launch_lines_1764},
    {1792, 16, 8, 14, 4, LinesCfg<Rad<16, 8, 14>, 4>::THREADS, LinesCfg<Rad<16, 8, 14>, 4>::SMEM_BYTES, launch_lines_1792},
    {1800, 15, 10, 12, 4, LinesCfg<Rad<15, 10, 12>, 4>::THREADS, LinesCfg<Rad<15, 10, 12>, 4>::SMEM_BYTES, launch_lines_1800},
    {1890, 15, 9, 14, 4, LinesCfg<Rad<15, 9, 14>, 4>::THREADS, LinesCfg<Rad<15, 9, 14>, 4>::SMEM_BYTES, launch_lines_1890},
    {1920, 16, 10, 12, 4, LinesCfg<Rad<16, 10, 12>, 4>::THREADS, LinesCfg<Rad<16, 10, 12>, 4>::SMEM_BYTES, launch_lines_1920},
    {1960, 14, 10, 14, 4, LinesCfg<Rad<14, 10, 14>, 4>::THREADS, LinesCfg<Rad<14, 10, 14>, 4>::SMEM_BYTES, launch_lines_1960},
    {2016, 14, 12, 12, 4, LinesCfg<Rad<14, 12, 12>, 4>::THREADS, LinesCfg<Rad<14, 12, 12>, 4>::SMEM_BYTES, launch_lines_2016},
    {2025, 15, 9, 15, 4, LinesCfg<Rad<15, 9, 15>, 4>::THREADS, LinesCfg<Rad<15, 9, 15>, 4>::SMEM_BYTES, launch_lines_2025},
    {2048, 16, 8, 16, 4, LinesCfg<Rad<16, 8, 16>, 4>::THREADS, LinesCfg<Rad<16, 8, 16>, 4>::SMEM_BYTES, launch_lines_2048},
    {2100, 15, 10, 14, 4, LinesCfg<Rad<15, 10, 14>, 4>::THREADS, LinesCfg<Rad<15, 10, 14>, 4>::SMEM_BYTES, launch_lines_2100},
    {2160, 15, 12, 12, 4, LinesCfg<Rad<15, 12, 12>, 4>::THREADS, LinesCfg<Rad<15, 12, 12>, 4>::SMEM_BYTES, launch_lines_2160},
    {2240, 16, 10, 14, 4, LinesCfg<Rad<16, 10, 14>, 4>::THREADS, LinesCfg<Rad<16, 10, 14>, 4>::SMEM_BYTES, launch_lines_2240},
    {2250, 15, 10, 15, 4, LinesCfg<Rad<15, 10, 15>, 4>::THREADS, LinesCfg<Rad<15, 10, 15>, 4>::SMEM_BYTES, launch_lines_2250},
    {2304, 16, 12, 12, 4, LinesCfg<Rad<16, 12, 12>, 4>::THREADS, LinesCfg<Rad<16, 12, 12>, 4>::SMEM_BYTES, launch_lines_2304},
    {2352, 14, 12, 14, 4, LinesCfg<Rad<14, 12, 14>, 4>::THREADS, LinesCfg<Rad<14, 12, 14>, 4>::SMEM_BYTES, launch_lines_2352},
    {2400, 16, 10, 15, 4, LinesCfg<Rad<16, 10, 15>, 4>::THREADS, LinesCfg<Rad<16, 10, 15>, 4>::SMEM_BYTES, launch_lines_2400},
    {2520, 15, 12, 14, 4, LinesCfg<Rad<15, 12, 14>, 4>::THREADS, LinesCfg<Rad<15, 12, 14>, 4>::SMEM_BYTES, launch_lines_2520},
    {2560, 16, 10, 16, 4, LinesCfg<Rad<16, 10, 16>, 4>::THREADS, LinesCfg<Rad<16, 10, 16>, 4>::SMEM_BYTES, launch_lines_2560},
    {2688, 16, 12, 14, 4, LinesCfg<Rad<16, 12, 14>, 4>::THREADS, LinesCfg<Rad<16, 12, 14>, 4>::SMEM_BYTES, launch_lines_2688},
    {2700, 15, 12, 15, 4, LinesCfg<Rad<15, 12, 15>, 4>::THREADS, LinesCfg<Rad<15, 12, 15>, 4>::SMEM_BYTES, launch_lines_2700},
    {2744, 14, 14, 14, 4, LinesCfg<Rad<14, 14, 14>, 4>::THREADS, LinesCfg<Rad<14, 14, 14>, 4>::SMEM_BYTES, launch_lines_2744},
    {2880, 16, 12, 15, 4, LinesCfg<Rad<16, 12, 15>, 4>::THREADS, LinesCfg<Rad<16, 12, 15>, 4>::SMEM_BYTES, launch_lines_2880},
    {2940, 15, 14, 14, 4, LinesCfg<Rad<15, 14, 14>, 4>::THREADS, LinesCfg<Rad<15, 14, 14>, 4>::SMEM_BYTES, launch_lines_2940},
    {3072, 16, 12, 16, 2, LinesCfg<Rad<16, 12, 16>, 2>::THREADS, LinesCfg<Rad<16, 12, 16>, 2>::SMEM_BYTES, launch_lines_3072},
    {3136, 16, 14, 14, 2, LinesCfg<Rad<16, 14, 14>, 2>::THREADS, LinesCfg<Rad<16, 14, 14>, 2>::SMEM_BYTES, launch_lines_3136},
    {3150, 15, 14, 15, 2, LinesCfg<Rad<15, 14, 15>, 2>::THREADS, LinesCfg<Rad<15, 14, 15>, 2>::SMEM_BYTES, launch_lines_3150},
    {3360, 16, 14, 15, 2, LinesCfg<Rad<16, 14, 15>, 2>::THREADS, LinesCfg<Rad<16, 14, 15>, 2>::SMEM_BYTES, launch_lines_3360},
    {3375, 15, 15, 15, 2, LinesCfg<Rad<15, 15, 15>, 2>::THREADS, LinesCfg<Rad<15, 15, 15>, 2>::SMEM_BYTES, launch_lines_3375},
    {3584, 16, 14, 16, 2, LinesCfg<Rad<16, 14, 16>, 2>::THREADS, LinesCfg<Rad<16, 14, 16>, 2>::SMEM_BYTES, launch_lines_3584},
    {3600, 16, 15, 15, 2, LinesCfg<Rad<16, 15, 15>, 2>::THREADS, LinesCfg<Rad<16, 15, 15>, 2>::SMEM_BYTES, launch_lines_3600},
    {3840, 16, 15, 16, 2, LinesCfg<Rad<16, 15, 16>, 2>::THREADS, LinesCfg<Rad<16, 15, 16>, 2>::SMEM_BYTES, launch_lines_3840},
    {4096, 16, 16, 16, 2, LinesCfg<Rad<16, 16, 16>, 2>::THREADS, LinesCfg<Rad<16, 16, 16>, 2>::SMEM_BYTES, launch_lines_4096},
};
static const XPlan kXPlans[] = {
    {2, 2, 1, 1, 32, XCfg<Rad<2, 1, 1>, 32>::THREADS, XCfg<Rad<2, 1, 1>, 32>::SMEM_BYTES, launch_x_2},
    {3, 3, 1, 1, 32, XCfg<Rad<3, 1, 1>, 32>::THREADS, XCfg<Rad<3, 1, 1>, 32>::SMEM_BYTES, launch_x_3},
    {4, 2, 2, 1, 32, XCfg<Rad<2, 2, 1>, 32>::THREADS, XCfg<Rad<2, 2, 1>, 32>::SMEM_BYTES, launch_x_4},
    {5, 5, 1, 1, 16, XCfg<Rad<5, 1, 1>, 16>::THREADS, XCfg<Rad<5, 1, 1>, 16>::SMEM_BYTES, launch_x_5},
    {6, 3, 2, 1, 32, XCfg<Rad<3, 2, 1>, 32>::THREADS, XCfg<Rad<3, 2, 1>, 32>::SMEM_BYTES, launch_x_6},
    {7, 7, 1, 1, 16, XCfg<Rad<7, 1, 1>, 16>::THREADS, XCfg<Rad<7, 1, 1>, 16>::SMEM_BYTES, launch_x_7},
    {8, 4, 2, 1, 16, XCfg<Rad<4, 2, 1>, 16>::THREADS, XCfg<Rad<4, 2, 1>, 16>::SMEM_BYTES, launch_x_8},
    {9, 3, 3, 1, 32, XCfg<Rad<3, 3, 1>, 32>::THREADS, XCfg<Rad<3, 3, 1>, 32>::SMEM_BYTES, launch_x_9},
    {10, 5, 2, 1, 16, XCfg<Rad<5, 2, 1>, 16>::THREADS, XCfg<Rad<5, 2, 1>, 16>::SMEM_BYTES, launch_x_10},
    {12, 4, 3, 1, 16, XCfg<Rad<4, 3, 1>, 16>::THREADS, XCfg<Rad<4, 3, 1>, 16>::SMEM_BYTES, launch_x_12},
    {14, 7, 2, 1, 16, XCfg<Rad<7, 2, 1>, 16>::THREADS, XCfg<Rad<7, 2, 1>, 16>::SMEM_BYTES, launch_x_14},
    {15, 5, 3, 1, 16, XCfg<Rad<5, 3, 1>, 16>::THREADS, XCfg<Rad<5, 3, 1>, 16>::SMEM_BYTES, launch_x_15},
    {16, 4, 4, 1, 16, XCfg<Rad<4, 4, 1>, 16>::THREADS, XCfg<Rad<4, 4, 1>, 16>::SMEM_BYTES, launch_x_16},
    {18, 6, 3, 1, 16, XCfg<Rad<6, 3, 1>, 16>::THREADS, XCfg<Rad<6, 3, 1>, 16>::SMEM_BYTES, launch_x_18},
    {20, 5, 4, 1, 16, XCfg<Rad<5, 4, 1>, 16>::THREADS, XCfg<Rad<5, 4, 1>, 16>::SMEM_BYTES, launch_x_20},
    {21, 7, 3, 1, 16, XCfg<Rad<7, 3, 1>, 16>::THREADS, XCfg<Rad<7, 3, 1>, 16>::SMEM_BYTES, launch_x_21},
    {24, 6, 4, 1, 16, XCfg<Rad<6, 4, 1>, 16>::THREADS, XCfg<Rad<6, 4, 1>, 16>::SMEM_BYTES, launch_x_24},
    {25, 5, 5, 1, 16, XCfg<Rad<5, 5, 1>, 16>::THREADS, XCfg<Rad<5, 5, 1>, 16>::SMEM_BYTES, launch_x_25},
    {27, 9, 3, 1, 8, XCfg<Rad<9, 3, 1>, 8>::THREADS, XCfg<Rad<9, 3, 1>, 8>::SMEM_BYTES, launch_x_27},
    {28, 7, 4, 1, 16, XCfg<Rad<7, 4, 1>, 16>::THREADS, XCfg<Rad<7, 4, 1>, 16>::SMEM_BYTES, launch_x_28},
    {30, 6, 5, 1, 16, XCfg<Rad<6, 5, 1>, 16>::THREADS, XCfg<Rad<6, 5, 1>, 16>::SMEM_BYTES, launch_x_30},
    {32, 8, 4, 1, 8, XCfg<Rad<8, 4, 1>, 8>::THREADS, XCfg<Rad<8, 4, 1>, 8>::SMEM_BYTES, launch_x_32},
    {35, 7, 5, 1, 16, XCfg<Rad<7, 5, 1>, 16>::THREADS, XCfg<Rad<7, 5, 1>, 16>::SMEM_BYTES, launch_x_35},
    {36, 6, 6, 1, 16, XCfg<Rad<6, 6, 1>, 16>::THREADS, XCfg<Rad<6, 6, 1>, 16>::SMEM_BYTES, launch_x_36},
    {40, 8, 5, 1, 8, XCfg<Rad<8, 5, 1>, 8>::THREADS, XCfg<Rad<8, 5, 1>, 8>::SMEM_BYTES, launch_x_40},
    {42, 7, 6, 1, 16, XCfg<Rad<7, 6, 1>, 16>::THREADS, XCfg<Rad<7, 6, 1>, 16>::SMEM_BYTES, launch_x_42},
    {45, 9, 5, 1, 8, XCfg<Rad<9, 5, 1>, 8>::THREADS, XCfg<Rad<9, 5, 1>, 8>::SMEM_BYTES, launch_x_45},
    {48, 8, 6, 1, 8, XCfg<Rad<8, 6, 1>, 8>::THREADS, XCfg<Rad<8, 6, 1>, 8>::SMEM_BYTES, launch_x_48},
    {49, 7, 7, 1, 16, XCfg<Rad<7, 7, 1>, 16>::THREADS, XCfg<Rad<7, 7, 1>, 16>::SMEM_BYTES, launch_x_49},
    {50, 10, 5, 1, 8, XCfg<Rad<10, 5, 1>, 8>::THREADS, XCfg<Rad<10, 5, 1>, 8>::SMEM_BYTES, launch_x_50},
    {54, 9, 6, 1, 8, XCfg<Rad<9, 6, 1>, 8>::THREADS, XCfg<Rad<9, 6, 1>, 8>::SMEM_BYTES, launch_x_54},
    {56, 8, 7, 1, 8, XCfg<Rad<8, 7, 1>, 8>::THREADS, XCfg<Rad<8, 7, 1>, 8>::SMEM_BYTES, launch_x_56},
    {60, 10, 6, 1, 8, XCfg<Rad<10, 6, 1>, 8>::THREADS, XCfg<Rad<10, 6, 1>, 8>::SMEM_BYTES, launch_x_60},
    {63, 9, 7, 1, 8, XCfg<Rad<9, 7, 1>, 8>::THREADS, XCfg<Rad<9, 7, 1>, 8>::SMEM_BYTES, launch_x_63},
    {64, 8, 8, 1, 8, XCfg<Rad<8, 8, 1>, 8>::THREADS, XCfg<Rad<8, 8, 1>, 8>::SMEM_BYTES, launch_x_64},
    {70, 10, 7, 1, 8, XCfg<Rad<10, 7, 1>, 8>::THREADS, XCfg<Rad<10, 7, 1>, 8>::SMEM_BYTES, launch_x_70},
    {72, 9, 8, 1, 8, XCfg<Rad<9, 8, 1>, 8>::THREADS, XCfg<Rad<9, 8, 1>, 8>::SMEM_BYTES, launch_x_72},
    {75, 15, 5, 1, 8, XCfg<Rad<15, 5, 1>, 8>::THREADS, XCfg<Rad<15, 5, 1>, 8>::SMEM_BYTES, launch_x_75},
    {80, 10, 8, 1, 8, XCfg<Rad<10, 8, 1>, 8>::THREADS, XCfg<Rad<10, 8, 1>, 8>::SMEM_BYTES, launch_x_80},
    {81, 9, 9, 1, 8, XCfg<Rad<9, 9, 1>, 8>::THREADS, XCfg<Rad<9, 9, 1>, 8>::SMEM_BYTES, launch_x_81},
    {84, 12, 7, 1, 8, XCfg<Rad<12, 7, 1>, 8>::THREADS, XCfg<Rad<12, 7, 1>, 8>::SMEM_BYTES, launch_x_84},
    {90, 10, 9, 1, 8, XCfg<Rad<10, 9, 1>, 8>::THREADS, XCfg<Rad<10, 9, 1>, 8>::SMEM_BYTES, launch_x_90},
    {96, 12, 8, 1, 8, XCfg<Rad<12, 8, 1>, 8>::THREADS, XCfg<Rad<12, 8, 1>, 8>::SMEM_BYTES, launch_x_96},
    {98, 14, 7, 1, 8, XCfg<Rad<14, 7, 1>, 8>::THREADS, XCfg<Rad<14, 7, 1>, 8>::SMEM_BYTES, launch_x_98},
    {100, 10, 10, 1, 8, XCfg<Rad<10, 10, 1>, 8>::THREADS, XCfg<Rad<10, 10, 1>, 8>::SMEM_BYTES, launch_x_100},
    {105, 15, 7, 1, 8, XCfg<Rad<15, 7, 1>, 8>::THREADS, XCfg<Rad<15, 7, 1>, 8>::SMEM_BYTES, launch_x_105},
    {108, 12, 9, 1, 8, XCfg<Rad<12, 9, 1>, 8>::THREADS, XCfg<Rad<12, 9, 1>, 8>::SMEM_BYTES, launch_x_108},
    {112, 14, 8, 1, 8, XCfg<Rad<14, 8, 1>, 8>::THREADS, XCfg<Rad<14, 8, 1>, 8>::SMEM_BYTES, launch_x_112},
    {120, 12, 10, 1, 8, XCfg<Rad<12, 10, 1>, 8>::THREADS, XCfg<Rad<12, 10, 1>, 8>::SMEM_BYTES, launch_x_120},
    {125, 5, 5, 5, 4, XCfg<Rad<5, 5, 5>, 4>::THREADS, XCfg<Rad<5, 5, 5>, 4>::SMEM_BYTES, launch_x_125},
    {126, 14, 9, 1, 8, XCfg<Rad<14, 9, 1>, 8>::THREADS, XCfg<Rad<14, 9, 1>, 8>::SMEM_BYTES, launch_x_126},
    {128, 16, 8, 1, 4, XCfg<Rad<16, 8, 1>, 4>::THREADS, XCfg<Rad<16, 8, 1>, 4>::SMEM_BYTES, launch_x_128},
    {135, 15, 9, 1, 8, XCfg<Rad<15, 9, 1>, 8>::THREADS, XCfg<Rad<15, 9, 1>, 8>::SMEM_BYTES, launch_x_135},
    {140, 14, 10, 1, 8, XCfg<Rad<14, 10, 1>, 8>::THREADS, XCfg<Rad<14, 10, 1>, 8>::SMEM_BYTES, launch_x_140},
    {144, 12, 12, 1, 8, XCfg<Rad<12, 12, 1>, 8>::THREADS, XCfg<Rad<12, 12, 1>, 8>::SMEM_BYTES, launch_x_144},
    {147, 7, 3, 7, 2, XCfg<Rad<7, 3, 7>, 2>::THREADS, XCfg<Rad<7, 3, 7>, 2>::SMEM_BYTES, launch_x_147},
    {150, 15, 10, 1, 8, XCfg<Rad<15, 10, 1>, 8>::THREADS, XCfg<Rad<15, 10, 1>, 8>::SMEM_BYTES, launch_x_150},
    {160, 16, 10, 1, 4, XCfg<Rad<16, 10, 1>, 4>::THREADS, XCfg<Rad<16, 10, 1>, 4>::SMEM_BYTES, launch_x_160},
    {162, 9, 3, 6, 2, XCfg<Rad<9, 3, 6>, 2>::THREADS, XCfg<Rad<9, 3, 6>, 2>::SMEM_BYTES, launch_x_162},
    {168, 14, 12, 1, 8, XCfg<Rad<14, 12, 1>, 8>::THREADS, XCfg<Rad<14, 12, 1>, 8>::SMEM_BYTES, launch_x_168},
    {175, 7, 5, 5, 2, XCfg<Rad<7, 5, 5>, 2>::THREADS, XCfg<Rad<7, 5, 5>, 2>::SMEM_BYTES, launch_x_175},
    {180, 15, 12, 1, 8, XCfg<Rad<15, 12, 1>, 8>::THREADS, XCfg<Rad<15, 12, 1>, 8>::SMEM_BYTES, launch_x_180},
    {189, 9, 3, 7, 2, XCfg<Rad<9, 3, 7>, 2>::THREADS, XCfg<Rad<9, 3, 7>, 2>::SMEM_BYTES, launch_x_189},
    {192, 16, 12, 1, 4, XCfg<Rad<16, 12, 1>, 4>::THREADS, XCfg<Rad<16, 12, 1>, 4>::SMEM_BYTES, launch_x_192},
    {196, 14, 14, 1, 8, XCfg<Rad<14, 14, 1>, 8>::THREADS, XCfg<Rad<14, 14, 1>, 8>::SMEM_BYTES, launch_x_196},
    {200, 8, 5, 5, 2, XCfg<Rad<8, 5, 5>, 2>::THREADS, XCfg<Rad<8, 5, 5>, 2>::SMEM_BYTES, launch_x_200},
    {210, 15, 14, 1, 8, XCfg<Rad<15, 14, 1>, 8>::THREADS, XCfg<Rad<15, 14, 1>, 8>::SMEM_BYTES, launch_x_210},
    {216, 6, 6, 6, 2, XCfg<Rad<6, 6, 6>, 2>::THREADS, XCfg<Rad<6, 6, 6>, 2>::SMEM_BYTES, launch_x_216},
    {224, 16, 14, 1, 4, XCfg<Rad<16, 14, 1>, 4>::THREADS, XCfg<Rad<16, 14, 1>, 4>::SMEM_BYTES, launch_x_224},
    {225, 15, 15, 1, 8, XCfg<Rad<15, 15, 1>, 8>::THREADS, XCfg<Rad<15, 15, 1>, 8>::SMEM_BYTES, launch_x_225},
    {240, 16, 15, 1, 4, XCfg<Rad<16, 15, 1>, 4>::THREADS, XCfg<Rad<16, 15, 1>, 4>::SMEM_BYTES, launch_x_240},
    {243, 9, 3, 9, 2, XCfg<Rad<9, 3, 9>, 2>::THREADS, XCfg<Rad<9, 3, 9>, 2>::SMEM_BYTES, launch_x_243},
    {245, 7, 5, 7, 2, XCfg<Rad<7, 5, 7>, 2>::THREADS, XCfg<Rad<7, 5, 7>, 2>::SMEM_BYTES, launch_x_245},
    {250, 10, 5, 5, 2, XCfg<Rad<10, 5, 5>, 2>::THREADS, XCfg<Rad<10, 5, 5>, 2>::SMEM_BYTES, launch_x_250},
    {252, 7, 6, 6, 2, XCfg<Rad<7, 6, 6>, 2>::THREADS, XCfg<Rad<7, 6, 6>, 2>::SMEM_BYTES, launch_x_252},
    {256, 16, 16, 1, 4, XCfg<Rad<16, 16, 1>, 4>::THREADS, XCfg<Rad<16, 16, 1>, 4>::SMEM_BYTES, launch_x_256},
    {270, 9, 5, 6, 2, XCfg<Rad<9, 5, 6>, 2>::THREADS, XCfg<Rad<9, 5, 6>, 2>::SMEM_BYTES, launch_x_270},
    {280, 8, 5, 7, 2, XCfg<Rad<8, 5, 7>, 2>::THREADS, XCfg<Rad<8, 5, 7>, 2>::SMEM_BYTES, launch_x_280},
    {288, 8, 6, 6, 2, XCfg<Rad<8, 6, 6>, 2>::THREADS, XCfg<Rad<8, 6, 6>, 2>::SMEM_BYTES, launch_x_288},
    {294, 7, 6, 7, 2, XCfg<Rad<7, 6, 7>, 2>::THREADS, XCfg<Rad<7, 6, 7>, 2>::SMEM_BYTES, launch_x_294},
    {300, 10, 5, 6, 2, XCfg<Rad<10, 5, 6>, 2>::THREADS, XCfg<Rad<10, 5, 6>, 2>::SMEM_BYTES, launch_x_300},
    {315, 9, 5, 7, 2, XCfg<Rad<9, 5, 7>, 2>::THREADS, XCfg<Rad<9, 5, 7>, 2>::SMEM_BYTES, launch_x_315},
    {320, 8, 5, 8, 2, XCfg<Rad<8, 5, 8>, 2>::THREADS, XCfg<Rad<8, 5, 8>, 2>::SMEM_BYTES, launch_x_320},
    {324, 9, 6, 6, 2, XCfg<Rad<9, 6, 6>, 2>::THREADS, XCfg<Rad<9, 6, 6>, 2>::SMEM_BYTES, launch_x_324},
    {336, 8, 6, 7, 2, XCfg<Rad<8, 6, 7>, 2>::THREADS, XCfg<Rad<8, 6, 7>, 2>::SMEM_BYTES, launch_x_336},
    {343, 7, 7, 7, 2, XCfg<Rad<7, 7, 7>, 2>::THREADS, XCfg<Rad<7, 7, 7>, 2>::SMEM_BYTES, launch_x_343},
    {350, 10, 5, 7, 2, XCfg<Rad<10, 5, 7>, 2>::THREADS, XCfg<Rad<10, 5, 7>, 2>::SMEM_BYTES, launch_x_350},
    {360, 10, 6, 6, 2, XCfg<Rad<10, 6, 6>, 2>::THREADS, XCfg<Rad<10, 6, 6>, 2>::SMEM_BYTES, launch_x_360},
    {375, 15, 5, 5, 2, XCfg<Rad<15, 5, 5>, 2>::THREADS, XCfg<Rad<15, 5, 5>, 2>::SMEM_BYTES, launch_x_375},
    {378, 9, 6, 7, 2, XCfg<Rad<9, 6, 7>, 2>::THREADS, XCfg<Rad<9, 6, 7>, 2>::SMEM_BYTES, launch_x_378},
    {384, 8, 6, 8, 2, XCfg<Rad<8, 6, 8>, 2>::THREADS, XCfg<Rad<8, 6, 8>, 2>::SMEM_BYTES, launch_x_384},
    {392, 8, 7, 7, 2, XCfg<Rad<8, 7, 7>, 2>::THREADS, XCfg<Rad<8, 7, 7>, 2>::SMEM_BYTES, launch_x_392},
    {400, 10, 5, 8, 2, XCfg<Rad<10, 5, 8>, 2>::THREADS, XCfg<Rad<10, 5, 8>, 2>::SMEM_BYTES, launch_x_400},
    {405, 9, 5, 9, 2, XCfg<Rad<9, 5, 9>, 2>::THREADS, XCfg<Rad<9, 5, 9>, 2>::SMEM_BYTES, launch_x_405},
    {420, 10, 6, 7, 2, XCfg<Rad<10, 6, 7>, 2>::THREADS, XCfg<Rad<10, 6, 7>, 2>::SMEM_BYTES, launch_x_420},
    {432, 9, 6, 8, 2, XCfg<Rad<9, 6, 8>, 2>::THREADS, XCfg<Rad<9, 6, 8>, 2>::SMEM_BYTES, launch_x_432},
    {441, 9, 7, 7, 2, XCfg<Rad<9, 7, 7>, 2>::THREADS, XCfg<Rad<9, 7, 7>, 2>::SMEM_BYTES, launch_x_441},
    {448, 8, 7, 8, 2, XCfg<Rad<8, 7, 8>, 2>::THREADS, XCfg<Rad<8, 7, 8>, 2>::SMEM_BYTES, launch_x_448},
    {450, 10, 5, 9, 2, XCfg<Rad<10, 5, 9>, 2>::THREADS, XCfg<Rad<10, 5, 9>, 2>::SMEM_BYTES, launch_x_450},
    {480, 10, 6, 8, 2, XCfg<Rad<10, 6, 8>, 2>::THREADS, XCfg<Rad<10, 6, 8>, 2>::SMEM_BYTES, launch_x_480},
    {486, 9, 6, 9, 2, XCfg<Rad<9, 6, 9>, 2>::THREADS, XCfg<Rad<9, 6, 9>, 2>::SMEM_BYTES, launch_x_486},
    {490, 10, 7, 7, 2, XCfg<Rad<10, 7, 7>, 2>::THREADS, XCfg<Rad<10, 7, 7>, 2>::SMEM_BYTES, launch_x_490},
    {500, 10, 5, 10, 2, XCfg<Rad<10, 5, 10>, 2>::THREADS, XCfg<Rad<10, 5, 10>, 2>::SMEM_BYTES, launch_x_500},
    {504, 9, 7, 8, 2, XCfg<Rad<9, 7, 8>, 2>::THREADS, XCfg<Rad<9, 7, 8>, 2>::SMEM_BYTES, launch_x_504},
    {512, 8, 8, 8, 2, XCfg<Rad<8, 8, 8>, 2>::THREADS, XCfg<Rad<8, 8, 8>, 2>::SMEM_BYTES, launch_x_512},
    {525, 15, 5, 7, 2, XCfg<Rad<15, 5, 7>, 2>::THREADS, XCfg<Rad<15, 5, 7>, 2>::SMEM_BYTES, launch_x_525},
    {540, 10, 6, 9, 2, XCfg<Rad<10, 6, 9>, 2>::THREADS, XCfg<Rad<10, 6, 9>, 2>::SMEM_BYTES, launch_x_540},
    {560, 10, 7, 8, 2, XCfg<Rad<10, 7, 8>, 2>::THREADS, XCfg<Rad<10, 7, 8>, 2>::SMEM_BYTES, launch_x_560},
    {567, 9, 7, 9, 2, XCfg<Rad<9, 7, 9>, 2>::THREADS, XCfg<Rad<9, 7, 9>, 2>::SMEM_BYTES, launch_x_567},
    {576, 9, 8, 8, 2, XCfg<Rad<9, 8, 8>, 2>::THREADS, XCfg<Rad<9, 8, 8>, 2>::SMEM_BYTES, launch_x_576},
    {588, 12, 7, 7, 2, XCfg<Rad<12, 7, 7>, 2>::THREADS, XCfg<Rad<12, 7, 7>, 2>::SMEM_BYTES, launch_x_588},
    {600, 10, 6, 10, 2, XCfg<Rad<10, 6, 10>, 2>::THREADS, XCfg<Rad<10, 6, 10>, 2>::SMEM_BYTES, launch_x_600},
    {630, 10, 7, 9, 2, XCfg<Rad<10, 7, 9>, 2>::THREADS, XCfg<Rad<10, 7, 9>, 2>::SMEM_BYTES, launch_x_630},
    {640, 10, 8, 8, 2, XCfg<Rad<10, 8, 8>, 2>::THREADS, XCfg<Rad<10, 8, 8>, 2>::SMEM_BYTES, launch_x_640},
    {648, 9, 8, 9, 2, XCfg<Rad<9, 8, 9>, 2>::THREADS, XCfg<Rad<9, 8, 9>, 2>::SMEM_BYTES, launch_x_648},
    {672, 12, 7, 8, 2, XCfg<Rad<12, 7, 8>, 2>::THREADS, XCfg<Rad<12, 7, 8>, 2>::SMEM_BYTES, launch_x_672},
    {675, 15, 5, 9, 2, XCfg<Rad<15, 5, 9>, 2>::THREADS, XCfg<Rad<15, 5, 9>, 2>::SMEM_BYTES, launch_x_675},
    {686, 14, 7, 7, 2, XCfg<Rad<14, 7, 7>, 2>::THREADS, XCfg<Rad<14, 7, 7>, 2>::SMEM_BYTES, launch_x_686},
    {700, 10, 7, 10, 2, XCfg<Rad<10, 7, 10>, 2>::THREADS, XCfg<Rad<10, 7, 10>, 2>::SMEM_BYTES, launch_x_700},
    {720, 10, 8, 9, 2, XCfg<Rad<10, 8, 9>, 2>::THREADS, XCfg<Rad<10, 8, 9>, 2>::SMEM_BYTES, launch_x_720},
    {729, 9, 9, 9, 2, XCfg<Rad<9, 9, 9>, 2>::THREADS, XCfg<Rad<9, 9, 9>, 2>::SMEM_BYTES, launch_x_729},
    {735, 15, 7, 7, 2, XCfg<Rad<15, 7, 7>, 2>::THREADS, XCfg<Rad<15, 7, 7>, 2>::SMEM_BYTES, launch_x_735},
    {750, 15, 5, 10, 2, XCfg<Rad<15, 5, 10>, 2>::THREADS, XCfg<Rad<15, 5, 10>, 2>::SMEM_BYTES, launch_x_750},
    {756, 12, 7, 9, 2, XCfg<Rad<12, 7, 9>, 2>::THREADS, XCfg<Rad<12, 7, 9>, 2>::SMEM_BYTES, launch_x_756},
    {768, 12, 8, 8, 2, XCfg<Rad<12, 8, 8>, 2>::THREADS, XCfg<Rad<12, 8, 8>, 2>::SMEM_BYTES, launch_x_768},
    {784, 14, 7, 8, 2, XCfg<Rad<14, 7, 8>, 2>::THREADS, XCfg<Rad<14, 7, 8>, 2>::SMEM_BYTES, launch_x_784},
    {800, 10, 8, 10, 2, XCfg<Rad<10, 8, 10>, 2>::THREADS, XCfg<Rad<10, 8, 10>, 2>::SMEM_BYTES, launch_x_800},
    {810, 10, 9, 9, 2, XCfg<Rad<10, 9, 9>, 2>::THREADS, XCfg<Rad<10, 9, 9>, 2>::SMEM_BYTES, launch_x_810},
    {840, 12, 7, 10, 2, XCfg<Rad<12, 7, 10>, 2>::THREADS, XCfg<Rad<12, 7, 10>, 2>::SMEM_BYTES, launch_x_840},
    {864, 12, 8, 9, 2, XCfg<Rad<12, 8, 9>, 2>::THREADS, XCfg<Rad<12, 8, 9>, 2>::SMEM_BYTES, launch_x_864},
    {882, 14, 7, 9, 2, XCfg<Rad<14, 7, 9>, 2>::THREADS, XCfg<Rad<14, 7, 9>, 2>::SMEM_BYTES, launch_x_882},
    {896, 14, 8, 8, 2, XCfg<Rad<14, 8, 8>, 2>::THREADS, XCfg<Rad<14, 8, 8>, 2>::SMEM_BYTES, launch_x_896},
    {900, 10, 9, 10, 2, XCfg<Rad<10, 9, 10>, 2>::THREADS, XCfg<Rad<10, 9, 10>, 2>::SMEM_BYTES, launch_x_900},
    {945, 15, 7, 9, 2, XCfg<Rad<15, 7, 9>, 2>::THREADS, XCfg<Rad<15, 7, 9>, 2>::SMEM_BYTES, launch_x_945},
    {960, 12, 8, 10, 2, XCfg<Rad<12, 8, 10>, 2>::THREADS, XCfg<Rad<12, 8, 10>, 2>::SMEM_BYTES, launch_x_960},
    {972, 12, 9, 9, 2, XCfg<Rad<12, 9, 9>, 2>::THREADS, XCfg<Rad<12, 9, 9>, 2>::SMEM_BYTES, launch_x_972},
    {980, 14, 7, 10, 2, XCfg<Rad<14, 7, 10>, 2>::THREADS, XCfg<Rad<14, 7, 10>, 2>::SMEM_BYTES, launch_x_980},
    {1000, 10, 10, 10, 2, XCfg<Rad<10, 10, 10>, 2>::THREADS, XCfg<Rad<10, 10, 10>, 2>::SMEM_BYTES, launch_x_1000},
    {1008, 14, 8, 9, 2, XCfg<Rad<14, 8, 9>, 2>::THREADS, XCfg<Rad<14, 8, 9>, 2>::SMEM_BYTES, launch_x_1008},
    {1024, 16, 8, 8, 2, XCfg<Rad<16, 8, 8>, 2>::THREADS, XCfg<Rad<16, 8, 8>, 2>::SMEM_BYTES, launch_x_1024},
    {1050, 15, 7, 10, 2, XCfg<Rad<15, 7, 10>, 2>::THREADS, XCfg<Rad<15, 7, 10>, 2>::SMEM_BYTES, launch_x_1050},
    {1080, 12, 9, 10, 2, XCfg<Rad<12, 9, 10>, 2>::THREADS, XCfg<Rad<12, 9, 10>, 2>::SMEM_BYTES, launch_x_1080},
    {1120, 14, 8, 10, 2, XCfg<Rad<14, 8, 10>, 2>::THREADS, XCfg<Rad<14, 8, 10>, 2>::SMEM_BYTES, launch_x_1120},
    {1125, 15, 5, 15, 1, XCfg<Rad<15, 5, 15>, 1>::THREADS, XCfg<Rad<15, 5, 15>, 1>::SMEM_BYTES, launch_x_1125},
    {1134, 14, 9, 9, 2, XCfg<Rad<14, 9, 9>, 2>::THREADS, XCfg<Rad<14, 9, 9>, 2>::SMEM_BYTES, launch_x_1134},
    {1152, 12, 8, 12, 1, XCfg<Rad<12, 8, 12>, 1>::THREADS, XCfg<Rad<12, 8, 12>, 1>::SMEM_BYTES, launch_x_1152},
    {1176, 14, 7, 12, 1, XCfg<Rad<14, 7, 12>, 1>::THREADS, XCfg<Rad<14, 7, 12>, 1>::SMEM_BYTES, launch_x_1176},
    {1200, 12, 10, 10, 1, XCfg<Rad<12, 10, 10>, 1>::THREADS, XCfg<Rad<12, 10, 10>, 1>::SMEM_BYTES, launch_x_1200},
    {1215, 15, 9, 9, 1, XCfg<Rad<15, 9, 9>, 1>::THREADS, XCfg<Rad<15, 9, 9>, 1>::SMEM_BYTES, launch_x_1215},
    {1260, 14, 9, 10, 1, XCfg<Rad<14, 9, 10>, 1>::THREADS, XCfg<Rad<14, 9, 10>, 1>::SMEM_BYTES, launch_x_1260},
    {1280, 16, 8, 10, 1, XCfg<Rad<16, 8, 10>, 1>::THREADS, XCfg<Rad<16, 8, 10>, 1>::SMEM_BYTES, launch_x_1280},
    {1296, 12, 9, 12, 1, XCfg<Rad<12, 9, 12>, 1>::THREADS, XCfg<Rad<12, 9, 12>, 1>::SMEM_BYTES, launch_x_1296},
    {1344, 14, 8, 12, 1, XCfg<Rad<14, 8, 12>, 1>::THREADS, XCfg<Rad<14, 8, 12>, 1>::SMEM_BYTES, launch_x_1344},
    {1350, 15, 9, 10, 1, XCfg<Rad<15, 9, 10>, 1>::THREADS, XCfg<Rad<15, 9, 10>, 1>::SMEM_BYTES, launch_x_1350},
    {1372, 14, 7, 14, 1, XCfg<Rad<14, 7, 14>, 1>::THREADS, XCfg<Rad<14, 7, 14>, 1>::SMEM_BYTES, launch_x_1372},
    {1400, 14, 10, 10, 1, XCfg<Rad<14, 10, 10>, 1>::THREADS, XCfg<Rad<14, 10, 10>, 1>::SMEM_BYTES, launch_x_1400},
    {1440, 12, 10, 12, 1, XCfg<Rad<12, 10, 12>, 1>::THREADS, XCfg<Rad<12, 10, 12>, 1>::SMEM_BYTES, launch_x_1440},
    {1470, 15, 7, 14, 1, XCfg<Rad<15, 7, 14>, 1>::THREADS, XCfg<Rad<15, 7, 14>, 1>::SMEM_BYTES, launch_x_1470},
    {1500, 15, 10, 10, 1, XCfg<Rad<15, 10, 10>, 1>::THREADS, XCfg<Rad<15, 10, 10>, 1>::SMEM_BYTES, launch_x_1500},
    {1512, 14, 9, 12, 1, XCfg<Rad<14, 9, 12>, 1>::THREADS, XCfg<Rad<14, 9, 12>, 1>::SMEM_BYTES, launch_x_1512},
    {1536, 16, 8, 12, 1, XCfg<Rad<16, 8, 12>, 1>::THREADS, XCfg<Rad<16, 8, 12>, 1>::SMEM_BYTES, launch_x_1536},
    {1568, 14, 8, 14, 1, XCfg<Rad<14, 8, 14>, 1>::THREADS, XCfg<Rad<14, 8, 14>, 1>::SMEM_BYTES, launch_x_1568},
    {1575, 15, 7, 15, 1, XCfg<Rad<15, 7, 15>, 1>::THREADS, XCfg<Rad<15, 7, 15>, 1>::SMEM_BYTES, launch_x_1575},
    {1600, 16, 10, 10, 1, XCfg<Rad<16, 10, 10>, 1>::THREADS, XCfg<Rad<16, 10, 10>, 1>::SMEM_BYTES, launch_x_1600},
    {1620, 15, 9, 12, 1, XCfg<Rad<15, 9, 12>, 1>::THREADS, XCfg<Rad<15, 9, 12>, 1>::SMEM_BYTES, launch_x_1620},
    {1680, 14, 10, 12, 1, XCfg<Rad<14, 10, 12>, 1>::THREADS, XCfg<Rad<14, 10, 12>, 1>::SMEM_BYTES, launch_x_1680},
    {1728, 12, 12, 12, 1, XCfg<Rad<12, 12, 12>, 1>::THREADS, XCfg<Rad<12, 12, 12>, 1>::SMEM_BYTES, launch_x_1728},
    {1764, 14, 9, 14, 1, XCfg<Rad<14, 9, 14>, 1>::THREADS, XCfg<Rad<14, 9, 14>, 1>::SMEM_BYTES, launch_x_1764},
    {1792, 16, 8, 14, 1, XCfg<Rad<16, 8, 14>, 1>::THREADS, XCfg<Rad<16, 8, 14>, 1>::SMEM_BYTES, launch_x_1792},
    {1800, 15, 10, 12, 1, XCfg<Rad<15, 10, 12>, 1>::THREADS, XCfg<Rad<15, 10, 12>, 1>::SMEM_BYTES, launch_x_1800},
    {1890, 15, 9, 14, 1, XCfg<Rad<15, 9, 14>, 1>::THREADS, XCfg<Rad<15, 9, 14>, 1>::SMEM_BYTES, launch_x_1890},
    {1920, 16, 10, 12, 1, XCfg<Rad<16, 10, 12>, 1>::THREADS, XCfg<Rad<16, 10, 12>, 1>::SMEM_BYTES, launch_x_1920},
    {1960, 14, 10, 14, 1, XCfg<Rad<14, 10, 14>, 1>::THREADS, XCfg<Rad<14, 10, 14>, 1>::SMEM_BYTES, launch_x_1960},
    {2016, 14, 12, 12, 1, XCfg<Rad<14, 12, 12>, 1>::THREADS, XCfg<Rad<14, 12, 12>, 1>::SMEM_BYTES, launch_x_2016},
    {2025, 15, 9, 15, 1, XCfg<Rad<15, 9, 15>, 1>::THREADS, XCfg<Rad<15, 9, 15>, 1>::SMEM_BYTES, launch_x_2025},
    {2048, 16, 8, 16, 1, XCfg<Rad<16, 8, 16>, 1>::THREADS, XCfg<Rad<16, 8, 16>, 1>::SMEM_BYTES, launch_x_2048},
};
static const YPlan kYPlans[] = {
    {2, 2, 1, 1, YCfg<Rad<2, 1, 1>>::THREADS, YCfg<Rad<2, 1, 1>>::SMEM_BYTES, launch_y_2},
    {3, 3, 1, 1, YCfg<Rad<3, 1, 1>>::THREADS, YCfg<Rad<3, 1, 1>>::SMEM_BYTES, launch_y_3},
    {4, 2, 2, 1, YCfg<Rad<2, 2, 1>>::THREADS, YCfg<Rad<2, 2, 1>>::SMEM_BYTES, launch_y_4},
    {5, 5, 1, 1, YCfg<Rad<5, 1, 1>>::THREADS, YCfg<Rad<5, 1, 1>>::SMEM_BYTES, launch_y_5},
    {6, 3, 2, 1, YCfg<Rad<3, 2, 1>>::THREADS, YCfg<Rad<3, 2, 1>>::SMEM_BYTES, launch_y_6},
    {7, 7, 1, 1, YCfg<Rad<7, 1, 1>>::THREADS, YCfg<Rad<7, 1, 1>>::SMEM_BYTES, launch_y_7},
    {8, 4, 2, 1, YCfg<Rad<4, 2, 1>>::THREADS, YCfg<Rad<4, 2, 1>>::SMEM_BYTES, launch_y_8},
    {9, 3, 3, 1, YCfg<Rad<3, 3, 1>>::THREADS, YCfg<Rad<3, 3, 1>>::SMEM_BYTES, launch_y_9},
    {10, 5, 2, 1, YCfg<Rad<5, 2, 1>>::THREADS, YCfg<Rad<5, 2, 1>>::SMEM_BYTES, launch_y_10},
    {12, 4, 3, 1, YCfg<Rad<4, 3, 1>>::THREADS, YCfg<Rad<4, 3, 1>>::SMEM_BYTES, launch_y_12},
    {14, 7, 2, 1, YCfg<Rad<7, 2, 1>>::THREADS, YCfg<Rad<7, 2, 1>>::SMEM_BYTES, launch_y_14},
    {15, 5, 3, 1, YCfg<Rad<5, 3, 1>>::THREADS, YCfg<Rad<5, 3, 1>>::SMEM_BYTES, launch_y_15},
    {16, 4, 4, 1, YCfg<Rad<4, 4, 1>>::THREADS, YCfg<Rad<4, 4, 1>>::SMEM_BYTES, launch_y_16},
    {18, 6, 3, 1, YCfg<Rad<6, 3, 1>>::THREADS, YCfg<Rad<6, 3, 1>>::SMEM_BYTES, launch_y_18},
    {20, 5, 4, 1, YCfg<Rad<5, 4, 1>>::THREADS, YCfg<Rad<5, 4, 1>>::SMEM_BYTES, launch_y_20},
    {21, 7, 3, 1, YCfg<Rad<7, 3, 1>>::THREADS, YCfg<Rad<7, 3, 1>>::SMEM_BYTES, launch_y_21},
    {24, 6, 4, 1, YCfg<Rad<6, 4, 1>>::THREADS, YCfg<Rad<6, 4, 1>>::SMEM_BYTES, launch_y_24},
    {25, 5, 5, 1, YCfg<Rad<5, 5, 1>>::THREADS, YCfg<Rad<5, 5, 1>>::SMEM_BYTES, launch_y_25},
    {27, 9, 3, 1, YCfg<Rad<9, 3, 1>>::THREADS, YCfg<Rad<9, 3, 1>>::SMEM_BYTES, launch_y_27},
    {28, 7, 4, 1, YCfg<Rad<7, 4, 1>>::THREADS, YCfg<Rad<7, 4, 1>>::SMEM_BYTES, launch_y_28},
    {30, 6, 5, 1, YCfg<Rad<6, 5, 1>>::THREADS, YCfg<Rad<6, 5, 1>>::SMEM_BYTES, launch_y_30},
    {32, 8, 4, 1, YCfg<Rad<8, 4, 1>>::THREADS, YCfg<Rad<8, 4, 1>>::SMEM_BYTES, launch_y_32},
    {35, 7, 5, 1, YCfg<Rad<7, 5, 1>>::THREADS, YCfg<Rad<7, 5, 1>>::SMEM_BYTES, launch_y_35},
    {36, 6, 6, 1, YCfg<Rad<6, 6, 1>>::THREADS, YCfg<Rad<6, 6, 1>>::SMEM_BYTES, launch_y_36},
    {40, 8, 5, 1, YCfg<Rad<8, 5, 1>>::THREADS, YCfg<Rad<8, 5, 1>>::SMEM_BYTES, launch_y_40},
    {42, 7, 6, 1, YCfg<Rad<7, 6, 1>>::THREADS, YCfg<Rad<7, 6, 1>>::SMEM_BYTES, launch_y_42},
    {45, 9, 5, 1, YCfg<Rad<9, 5, 1>>::THREADS, YCfg<Rad<9, 5, 1>>::SMEM_BYTES, launch_y_45},
    {48, 8, 6, 1, YCfg<Rad<8, 6, 1>>::THREADS, YCfg<Rad<8, 6, 1>>::SMEM_BYTES, launch_y_48},
    {49, 7, 7, 1, YCfg<Rad<7, 7, 1>>::THREADS, YCfg<Rad<7, 7, 1>>::SMEM_BYTES, launch_y_49},
    {50, 10, 5, 1, YCfg<Rad<10, 5, 1>>::THREADS, YCfg<Rad<10, 5, 1>>::SMEM_BYTES, launch_y_50},
    {54, 9, 6, 1, YCfg<Rad<9, 6, 1>>::THREADS, YCfg<Rad<9, 6, 1>>::SMEM_BYTES, launch_y_54},
    {56, 8, 7, 1, YCfg<Rad<8, 7, 1>>::THREADS, YCfg<Rad<8, 7, 1>>::SMEM_BYTES, launch_y_56},
    {60, 10, 6, 1, YCfg<Rad<10, 6, 1>>::THREADS, YCfg<Rad<10, 6, 1>>::SMEM_BYTES, launch_y_60},
    {63, 9, 7, 1, YCfg<Rad<9, 7, 1>>::THREADS, YCfg<Rad<9, 7, 1>>::SMEM_BYTES, launch_y_63},
    {64, 8, 8, 1, YCfg<Rad<8, 8, 1>>::THREADS, YCfg<Rad<8, 8, 1>>::SMEM_BYTES, launch_y_64},
    {70, 10, 7, 1, YCfg<Rad<10, 7, 1>>::THREADS, YCfg<Rad<10, 7, 1>>::SMEM_BYTES, launch_y_70},
    {72, 9, 8, 1, YCfg<Rad<9, 8, 1>>::THREADS, YCfg<Rad<9, 8, 1>>::SMEM_BYTES, launch_y_72},
    {75, 15, 5, 1, YCfg<Rad<15, 5, 1>>::THREADS, YCfg<Rad<15, 5, 1>>::SMEM_BYTES, launch_y_75},
    {80, 10, 8, 1, YCfg<Rad<10, 8, 1>>::THREADS, YCfg<Rad<10, 8, 1>>::SMEM_BYTES, launch_y_80},
    {81, 9, 9, 1, YCfg<Rad<9, 9, 1>>::THREADS, YCfg<Rad<9, 9, 1>>::SMEM_BYTES, launch_y_81},
    {84, 12, 7, 1, YCfg<Rad<12, 7, 1>>::THREADS, YCfg<Rad<12, 7, 1>>::SMEM_BYTES, launch_y_84},
    {90, 10, 9, 1, YCfg<Rad<10, 9, 1>>::THREADS, YCfg<Rad<10, 9, 1>>::SMEM_BYTES, launch_y_90},
    {96, 12, 8, 1, YCfg<Rad<12, 8, 1>>::THREADS, YCfg<Rad<12, 8, 1>>::SMEM_BYTES, launch_y_96},
    {98, 14, 7, 1, YCfg<Rad<14, 7, 1>>::THREADS, YCfg<Rad<14, 7, 1>>::SMEM_BYTES, launch_y_98},
    {100, 10, 10, 1, YCfg<Rad<10, 10, 1>>::THREADS, YCfg<Rad<10, 10, 1>>::SMEM_BYTES, launch_y_100},
    {105, 15, 7, 1, YCfg<Rad<15, 7, 1>>::THREADS, YCfg<Rad<15, 7, 1>>::SMEM_BYTES, launch_y_105},
    {108, 12, 9, 1, YCfg<Rad<12, 9, 1>>::THREADS, YCfg<Rad<12, 9, 1>>::SMEM_BYTES, launch_y_108},
    {112, 14, 8, 1, YCfg<Rad<14, 8, 1>>::THREADS, YCfg<Rad<14, 8, 1>>::SMEM_BYTES, launch_y_112},
    {120, 12, 10, 1, YCfg<Rad<12, 10, 1>>::THREADS, YCfg<Rad<12, 10, 1>>::SMEM_BYTES, launch_y_120},
    {125, 5, 5, 5, YCfg<Rad<5, 5, 5>>::THREADS, YCfg<Rad<5, 5, 5>>::SMEM_BYTES, launch_y_125},
    {126, 14, 9, 1, YCfg<Rad<14, 9, 1>>::THREADS, YCfg<Rad<14, 9, 1>>::SMEM_BYTES, launch_y_126},
    {128, 16, 8, 1, YCfg<Rad<16, 8, 1>>::THREADS, YCfg<Rad<16, 8, 1>>::SMEM_BYTES, launch_y_128},
    {135, 15, 9, 1, YCfg<Rad<15, 9, 1>>::THREADS, YCfg<Rad<15, 9, 1>>::SMEM_BYTES, launch_y_135},
    {140, 14, 10, 1, YCfg<Rad<14, 10, 1>>::THREADS, YCfg<Rad<14, 10, 1>>::SMEM_BYTES, launch_y_140},
    {144, 12, 12, 1, YCfg<Rad<12, 12, 1>>::THREADS, YCfg<Rad<12, 12, 1>>::SMEM_BYTES, launch_y_144},
    {147, 7, 3, 7, YCfg<Rad<7, 3, 7>>::THREADS, YCfg<Rad<7, 3, 7>>::SMEM_BYTES, launch_y_147},
    {150, 15, 10, 1, YCfg<Rad<15, 10, 1>>::THREADS, YCfg<Rad<15, 10, 1>>::SMEM_BYTES, launch_y_150},
    {160, 16, 10, 1, YCfg<Rad<16, 10, 1>>::THREADS, YCfg<Rad<16, 10, 1>>::SMEM_BYTES, launch_y_160},
    {162, 9, 3, 6, YCfg<Rad<9, 3, 6>>::THREADS, YCfg<Rad<9, 3, 6>>::SMEM_BYTES, launch_y_162},
    {168, 14, 12, 1, YCfg<Rad<14, 12, 1>>::THREADS, YCfg<Rad<14, 12, 1>>::SMEM_BYTES, launch_y_168},
    {175, 7, 5, 5, YCfg<Rad<7, 5, 5>>::THREADS, YCfg<Rad<7, 5, 5>>::SMEM_BYTES, launch_y_175},
    {180, 15, 12, 1, YCfg<Rad<15, 12, 1>>::THREADS, YCfg<Rad<15, 12, 1>>::SMEM_BYTES, launch_y_180},
    {189, 9, 3, 7, YCfg<Rad<9, 3, 7>>::THREADS, YCfg<Rad<9, 3, 7>>::SMEM_BYTES, launch_y_189},
    {192, 16, 12, 1, YCfg<Rad<16, 12, 1>>::THREADS, YCfg<Rad<16, 12, 1>>::SMEM_BYTES, launch_y_192},
    {196, 14, 14, 1, YCfg<Rad<14, 14, 1>>::THREADS, YCfg<Rad<14, 14, 1>>::SMEM_BYTES, launch_y_196},
    {200, 8, 5, 5, YCfg<Rad<8, 5, 5>>::THREADS, YCfg<Rad<8, 5, 5>>::SMEM_BYTES, launch_y_200},
    {210, 15, 14, 1, YCfg<Rad<15, 14, 1>>::THREADS, YCfg<Rad<15, 14, 1>>::SMEM_BYTES, launch_y_210},
    {216, 6, 6, 6, YCfg<Rad<6, 6, 6>>::THREADS, YCfg<Rad<6, 6, 6>>::SMEM_BYTES, launch_y_216},
    {224, 16, 14, 1, YCfg<Rad<16, 14, 1>>::THREADS, YCfg<Rad<16, 14, 1>>::SMEM_BYTES, launch_y_224},
    {225, 15, 15, 1, YCfg<Rad<15, 15, 1>>::THREADS, YCfg<Rad<15, 15, 1>>::SMEM_BYTES, launch_y_225},
    {240, 16, 15, 1, YCfg<Rad<16, 15, 1>>::THREADS, YCfg<Rad<16, 15, 1>>::SMEM_BYTES, launch_y_240},
    {243, 9, 3, 9, YCfg<Rad<9, 3, 9>>::THREADS, YCfg<Rad<9, 3, 9>>::SMEM_BYTES, launch_y_243},
    {245, 7, 5, 7, YCfg<Rad<7, 5, 7>>::THREADS, YCfg<Rad<7, 5, 7>>::SMEM_BYTES, launch_y_245},
    {250, 10, 5, 5, YCfg<Rad<10, 5, 5>>::THREADS, YCfg<Rad<10, 5, 5>>::SMEM_BYTES, launch_y_250},
    {252, 7, 6, 6, YCfg<Rad<7, 6, 6>>::THREADS, YCfg<Rad<7, 6, 6>>::SMEM_BYTES, launch_y_252},
    {256, 16, 16, 1, YCfg<Rad<16, 16, 1>>::THREADS, YCfg<Rad<16, 16, 1>>::SMEM_BYTES, launch_y_256},
    {270, 9, 5, 6, YCfg<Rad<9, 5, 6>>::THREADS, YCfg<Rad<9, 5, 6>>::SMEM_BYTES, launch_y_270},
    {280, 8, 5, 7, YCfg<Rad<8, 5, 7>>::THREADS, YCfg<Rad<8, 5, 7>>::SMEM_BYTES, launch_y_280},
    {288, 8, 6, 6, YCfg<Rad<8, 6, 6>>::THREADS, YCfg<Rad<8, 6, 6>>::SMEM_BYTES, launch_y_288},
    {294, 7, 6, 7, YCfg<Rad<7, 6, 7>>::THREADS, YCfg<Rad<7, 6, 7>>::SMEM_BYTES, launch_y_294},
    {300, 10, 5, 6, YCfg<Rad<10, 5, 6>>::THREADS, YCfg<Rad<10, 5, 6>>::SMEM_BYTES, launch_y_300},
    {315, 9, 5, 7, YCfg<Rad<9, 5, 7>>::THREADS, YCfg<Rad<9, 5, 7>>::SMEM_BYTES, launch_y_315},
    {320, 8, 5, 8, YCfg<Rad<8, 5, 8>>::THREADS, YCfg<Rad<8, 5, 8>>::SMEM_BYTES, launch_y_320},
    {324, 9, 6, 6, YCfg<Rad<9, 6, 6>>::THREADS, YCfg<Rad<9, 6, 6>>::SMEM_BYTES, launch_y_324},
    {336, 8, 6, 7, YCfg<Rad<8, 6, 7>>::THREADS, YCfg<Rad<8, 6, 7>>::SMEM_BYTES, launch_y_336},
    {343, 7, 7, 7, YCfg<Rad<7, 7, 7>>::THREADS, YCfg<Rad<7, 7, 7>>::SMEM_BYTES, launch_y_343},
    {350, 10, 5, 7, YCfg<Rad<10, 5, 7>>::THREADS, YCfg<Rad<10, 5, 7>>::SMEM_BYTES, launch_y_350},
    {360, 10, 6, 6, YCfg<Rad<10, 6, 6>>::THREADS, YCfg<Rad<10, 6, 6>>::SMEM_BYTES, launch_y_360},
    {375, 15, 5, 5, YCfg<Rad<15, 5, 5>>::THREADS, YCfg<Rad<15, 5, 5>>::SMEM_BYTES, launch_y_375},
    {378, 9, 6, 7, YCfg<Rad<9, 6, 7>>::THREADS, YCfg<Rad<9, 6, 7>>::SMEM_BYTES, launch_y_378},
    {384, 8, 6, 8, YCfg<Rad<8, 6, 8>>::THREADS, YCfg<Rad<8, 6, 8>>::SMEM_BYTES, launch_y_384},
    {392, 8, 7, 7, YCfg<Rad<8, 7, 7>>::THREADS, YCfg<Rad<8, 7, 7>>::SMEM_BYTES, launch_y_392},
    {400, 10, 5, 8, YCfg<Rad<10, 5, 8>>::THREADS, YCfg<Rad<10, 5, 8>>::SMEM_BYTES, launch_y_400},
    {405, 9, 5, 9, YCfg<Rad<9, 5, 9>>::THREADS, YCfg<Rad<9, 5, 9>>::SMEM_BYTES, launch_y_405},
    {420, 10, 6, 7, YCfg<Rad<10, 6, 7>>::THREADS, YCfg<Rad<10, 6, 7>>::SMEM_BYTES, launch_y_420},
    {432, 9, 6, 8, YCfg<Rad<9, 6, 8>>::THREADS, YCfg<Rad<9, 6, 8>>::SMEM_BYTES, launch_y_432},
    {441, 9, 7, 7, YCfg<Rad<9, 7, 7>>::THREADS, YCfg<Rad<9, 7, 7>>::SMEM_BYTES, launch_y_441},
    {448, 8, 7, 8, YCfg<Rad<8, 7, 8>>::THREADS, YCfg<Rad<8, 7, 8>>::SMEM_BYTES, launch_y_448},
    {450, 10, 5, 9, YCfg<Rad<10, 5, 9>>::THREADS, YCfg<Rad<10, 5, 9>>::SMEM_BYTES, launch_y_450},
    {480, 10, 6, 8, YCfg<Rad<10, 6, 8>>::THREADS, YCfg<Rad<10, 6, 8>>::SMEM_BYTES, launch_y_480},
    {486, 9, 6, 9, YCfg<Rad<9, 6, 9>>::THREADS, YCfg<Rad<9, 6, 9>>::SMEM_BYTES, launch_y_486},
    {490, 10, 7, 7, YCfg<Rad<10, 7, 7>>::THREADS, YCfg<Rad<10, 7, 7>>::SMEM_BYTES, launch_y_490},
    {500, 10, 5, 10, YCfg<Rad<10, 5, 10>>::THREADS, YCfg<Rad<10, 5, 10>>::SMEM_BYTES, launch_y_500},
    {504, 9, 7, 8, YCfg<Rad<9, 7, 8>>::THREADS, YCfg<Rad<9, 7, 8>>::SMEM_BYTES, launch_y_504},
    {512, 8, 8, 8, YCfg<Rad<8, 8, 8>>::THREADS, YCfg<Rad<8, 8, 8>>::SMEM_BYTES, launch_y_512},
    {525, 15, 5, 7, YCfg<Rad<15, 5, 7>>::THREADS, YCfg<Rad<15, 5, 7>>::SMEM_BYTES, launch_y_525},
    {540, 10, 6, 9, YCfg<Rad<10, 6, 9>>::THREADS, YCfg<Rad<10, 6, 9>>::SMEM_BYTES, launch_y_540},
    {560, 10, 7, 8, YCfg<Rad<10, 7, 8>>::THREADS, YCfg<Rad<10, 7, 8>>::SMEM_BYTES, launch_y_560},
    {567, 9, 7, 9, YCfg<Rad<9, 7, 9>>::THREADS, YCfg<Rad<9, 7, 9>>::SMEM_BYTES, launch_y_567},
    {576, 9, 8, 8, YCfg<Rad<9, 8, 8>>::THREADS, YCfg<Rad<9, 8, 8>>::SMEM_BYTES, launch_y_576},
    {588, 12, 7, 7, YCfg<Rad<12, 7, 7>>::THREADS, YCfg<Rad<12, 7, 7>>::SMEM_BYTES, launch_y_588},
    {600, 10, 6, 10, YCfg<Rad<10, 6, 10>>::THREADS, YCfg<Rad<10, 6, 10>>::SMEM_BYTES, launch_y_600},
    {630, 10, 7, 9, YCfg<Rad<10, 7, 9>>::THREADS, YCfg<Rad<10, 7, 9>>::SMEM_BYTES, launch_y_630},
    {640, 10, 8, 8, YCfg<Rad<10, 8, 8>>::THREADS, YCfg<Rad<10, 8, 8>>::SMEM_BYTES, launch_y_640},
    {648, 9, 8, 9, YCfg<Rad<9, 8, 9>>::THREADS, YCfg<Rad<9, 8, 9>>::SMEM_BYTES, launch_y_648},
    {672, 12, 7, 8, YCfg<Rad<12, 7, 8>>::THREADS, YCfg<Rad<12, 7, 8>>::SMEM_BYTES, launch_y_672},
    {675, 15, 5, 9, YCfg<Rad<15, 5, 9>>::THREADS, YCfg<Rad<15, 5, 9>>::SMEM_BYTES, launch_y_675},
    {686, 14, 7, 7, YCfg<Rad<14, 7, 7>>::THREADS, YCfg<Rad<14, 7, 7>>::SMEM_BYTES, launch_y_686},
    {700, 10, 7, 10, YCfg<Rad<10, 7, 10>>::THREADS, YCfg<Rad<10, 7, 10>>::SMEM_BYTES, launch_y_700},
    {720, 10, 8, 9, YCfg<Rad<10, 8, 9>>::THREADS, YCfg<Rad<10, 8, 9>>::SMEM_BYTES, launch_y_720},
    {729, 9, 9, 9, YCfg<Rad<9, 9, 9>>::THREADS, YCfg<Rad<9, 9, 9>>::SMEM_BYTES, launch_y_729},
    {735, 15, 7, 7, YCfg<Rad<15, 7, 7>>::THREADS, YCfg<Rad<15, 7, 7>>::SMEM_BYTES, launch_y_735},
    {750, 15, 5, 10, YCfg<Rad<15, 5, 10>>::THREADS, YCfg<Rad<15, 5, 10>>::SMEM_BYTES, launch_y_750},
    {756, 12, 7, 9, YCfg<Rad<12, 7, 9>>::THREADS, YCfg<Rad<12, 7, 9>>::SMEM_BYTES, launch_y_756},
    {768, 12, 8, 8, YCfg<Rad<12, 8, 8>>::THREADS, YCfg<Rad<12, 8, 8>>::SMEM_BYTES, launch_y_768},
    {784, 14, 7, 8, YCfg<Rad<14, 7, 8>>::THREADS, YCfg<Rad<14, 7, 8>>::SMEM_BYTES, launch_y_784},
    {800, 10, 8, 10, YCfg<Rad<10, 8, 10>>::THREADS, YCfg<Rad<10, 8, 10>>::SMEM_BYTES, launch_y_800},
    {810, 10, 9, 9, YCfg<Rad<10, 9, 9>>::THREADS, YCfg<Rad<10, 9, 9>>::SMEM_BYTES, launch_y_810},
    {840, 12, 7, 10, YCfg<Rad<12, 7, 10>>::THREADS, YCfg<Rad<12, 7, 10>>::SMEM_BYTES, launch_y_840},
    {864, 12, 8, 9, YCfg<Rad<12, 8, 9>>::THREADS, YCfg<Rad<12, 8, 9>>::SMEM_BYTES, launch_y_864},
    {882, 14, 7, 9, YCfg<Rad<14, 7, 9>>::THREADS, YCfg<Rad<14, 7, 9>>::SMEM_BYTES, launch_y_882},
    {896, 14, 8, 8, YCfg<Rad<14, 8, 8>>::THREADS, YCfg<Rad<14, 8, 8>>::SMEM_BYTES, launch_y_896},
    {900, 10, 9, 10, YCfg<Rad<10, 9, 10>>::THREADS, YCfg<Rad<10, 9, 10>>::SMEM_BYTES, launch_y_900},
    {945, 15, 7, 9, YCfg<Rad<15, 7, 9>>::THREADS, YCfg<Rad<15, 7, 9>>::SMEM_BYTES, launch_y_945},
    {960, 12, 8, 10, YCfg<Rad<12, 8, 10>>::THREADS, YCfg<Rad<12, 8, 10>>::SMEM_BYTES, launch_y_960},
    {972, 12, 9, 9, YCfg<Rad<12, 9, 9>>::THREADS, YCfg<Rad<12, 9, 9>>::SMEM_BYTES, launch_y_972},
    {980, 14, 7, 10, YCfg<Rad<14, 7, 10>>::THREADS, YCfg<Rad<14, 7, 10>>::SMEM_BYTES, launch_y_980},
    {1000, 10, 10, 10, YCfg<Rad<10, 10, 10>>::THREADS, YCfg<Rad<10, 10, 10>>::SMEM_BYTES, launch_y_1000},
    {1008, 14, 8, 9, YCfg<Rad<14, 8, 9>>::THREADS, YCfg<Rad<14, 8, 9>>::SMEM_BYTES, launch_y_1008},
    {1024, 16, 8, 8, YCfg<Rad<16, 8, 8>>::THREADS, YCfg<Rad<16, 8, 8>>::SMEM_BYTES, launch_y_1024},
    {1050, 15, 7, 10, YCfg<Rad<15, 7, 10>>::THREADS, YCfg<Rad<15, 7, 10>>::SMEM_BYTES, launch_y_1050},
    {1080, 12, 9, 10, YCfg<Rad<12, 9, 10>>::THREADS, YCfg<Rad<12, 9, 10>>::SMEM_BYTES, launch_y_1080},
    {1120, 14, 8, 10, YCfg<Rad<14, 8, 10>>::THREADS, YCfg<Rad<14, 8, 10>>::SMEM_BYTES, launch_y_1120},
    {1125, 15, 5, 15, YCfg<Rad<15, 5, 15>>::THREADS, YCfg<Rad<15, 5, 15>>::SMEM_BYTES, launch_y_1125},
    {1134, 14, 9, 9, YCfg<Rad<14, 9, 9>>::THREADS, YCfg<Rad<14, 9, 9>>::SMEM_BYTES, launch_y_1134},
    {1152, 12, 8, 12, YCfg<Rad<12, 8, 12>>::THREADS, YCfg<Rad<12, 8, 12>>::SMEM_BYTES, launch_y_1152},
    {1176, 14, 7, 12, YCfg<Rad<14, 7, 12>>::THREADS, YCfg<Rad<14, 7, 12>>::SMEM_BYTES, launch_y_1176},
    {1200, 12, 10, 10, YCfg<Rad<12, 10, 10>>::THREADS, YCfg<Rad<12, 10, 10>>::SMEM_BYTES, launch_y_1200},
    {1215, 15, 9, 9, YCfg<Rad<15, 9, 9>>::THREADS, YCfg<Rad<15, 9, 9>>::SMEM_BYTES, launch_y_1215},
    {1260, 14, 9, 10, YCfg<Rad<14, 9, 10>>::THREADS, YCfg<Rad<14, 9, 10>>::SMEM_BYTES, launch_y_1260},
    {1280, 16, 8, 10, YCfg<Rad<16, 8, 10>>::THREADS, YCfg<Rad<16, 8, 10>>::SMEM_BYTES, launch_y_1280},
    {1296, 12, 9, 12, YCfg<Rad<12, 9, 12>>::THREADS, YCfg<Rad<12, 9, 12>>::SMEM_BYTES, launch_y_1296},
    {1344, 14, 8, 12, YCfg<Rad<14, 8, 12>>::THREADS, YCfg<Rad<14, 8, 12>>::SMEM_BYTES, launch_y_1344},
    {1350, 15, 9, 10, YCfg<Rad<15, 9, 10>>::THREADS, YCfg<Rad<15, 9, 10>>::SMEM_BYTES, launch_y_1350},
    {1372, 14, 7, 14, YCfg<Rad<14, 7, 14>>::THREADS, YCfg<Rad<14, 7, 14>>::SMEM_BYTES, launch_y_1372},
    {1400, 14, 10, 10, YCfg<Rad<14, 10, 10>>::THREADS, YCfg<Rad<14, 10, 10>>::SMEM_BYTES, launch_y_1400},
    {1440, 12, 10, 12, YCfg<Rad<12, 10, 12>>::THREADS, YCfg<Rad<12, 10, 12>>::SMEM_BYTES, launch_y_1440},
    {1470, 15, 7, 14, YCfg<Rad<15, 7, 14>>::THREADS, YCfg<Rad<15, 7, 14>>::SMEM_BYTES, launch_y_1470},
    {1500, 15, 10, 10, YCfg<Rad<15, 10, 10>>::THREADS, YCfg<Rad<15, 10, 10>>::SMEM_BYTES, launch_y_1500},
    {1512, 14, 9, 12, YCfg<Rad<14, 9, 12>>::THREADS, YCfg<Rad<14, 9, 12>>::SMEM_BYTES, launch_y_1512},
    {1536, 16, 8, 12, YCfg<Rad<16, 8, 12>>::THREADS, YCfg<Rad<16, 8, 12>>::SMEM_BYTES, launch_y_1536},
    {1568, 14, 8, 14, YCfg<Rad<14, 8, 14>>::THREADS, YCfg<Rad<14, 8, 14>>::SMEM_BYTES, launch_y_1568},
    {1575, 15, 7, 15, YCfg<Rad<15, 7, 15>>::THREADS, YCfg<Rad<15, 7, 15>>::SMEM_BYTES, launch_y_1575},
    {1600, 16, 10, 10, YCfg<Rad<16, 10, 10>>::THREADS, YCfg<Rad<16, 10, 10>>::SMEM_BYTES, launch_y_1600},
    {1620, 15, 9, 12, YCfg<Rad<15, 9, 12>>::THREADS, YCfg<Rad<15, 9, 12>>::SMEM_BYTES, launch_y_1620},
    {1680, 14, 10, 12, YCfg<Rad<14, 10, 12>>::THREADS, YCfg<Rad<14, 10, 12>>::SMEM_BYTES, launch_y_1680},
    {1728, 12, 12, 12, YCfg<Rad<12, 12, 12>>::THREADS, YCfg<Rad<12, 12, 12>>::SMEM_BYTES, launch_y_1728},
    {1764, 14, 9, 14, YCfg<Rad<14, 9, 14>>::THREADS, YCfg<Rad<14, 9, 14>>::SMEM_BYTES, launch_y_1764},
    {1792, 16, 8, 14, YCfg<Rad<16, 8, 14>>::THREADS, YCfg<Rad<16, 8, 14>>::SMEM_BYTES, launch_y_1792},
    {1800, 15, 10, 12, YCfg<Rad<15, 10, 12>>::THREADS, YCfg<Rad<15, 10, 12>>::SMEM_BYTES, launch_y_1800},
    {1890, 15, 9, 14, YCfg<Rad<15, 9, 14>>::THREADS, YCfg<Rad<15, 9, 14>>::SMEM_BYTES, launch_y_1890},
    {1920, 16, 10, 12, YCfg<Rad<16, 10, 12>>::THREADS, YCfg<Rad<16, 10, 12>>::SMEM_BYTES, launch_y_1920},
    {1960, 14, 10, 14, YCfg<Rad<14, 10, 14>>::THREADS, YCfg<Rad<14, 10, 14>>::SMEM_BYTES, launch_y_1960},
    {2016, 14, 12, 12, YCfg<Rad<14, 12, 12>>::THREADS, YCfg<Rad<14, 12, 12>>::SMEM_BYTES, launch_y_2016},
    {2025, 15, 9, 15, YCfg<Rad<15, 9, 15>>::THREADS, YCfg<Rad<15, 9, 15>>::SMEM_BYTES, launch_y_2025},
    {2048, 16, 8, 16, YCfg<Rad<16, 8, 16>>::THREADS, YCfg<Rad<16, 8, 16>>::SMEM_BYTES, launch_y_2048},
    {2100, 15, 10, 14, YCfg<Rad<15, 10, 14>>::THREADS, YCfg<Rad<15, 10, 14>>::SMEM_BYTES, launch_y_2100},
    {2160, 15, 12, 12, YCfg<Rad<15, 12, 12>>::THREADS, YCfg<Rad<15, 12, 12>>::SMEM_BYTES, launch_y_2160},
    {2240, 16, 10, 14, YCfg<Rad<16, 10, 14>>::THREADS, YCfg<Rad<16, 10, 14>>::SMEM_BYTES, launch_y_2240},
    {2250, 15, 10, 15, YCfg<Rad<15, 10, 15>>::THREADS, YCfg<Rad<15, 10, 15>>::SMEM_BYTES, launch_y_2250},
    {2304, 16, 12, 12, YCfg<Rad<16, 12, 12>>::THREADS, YCfg<Rad<16, 12, 12>>::SMEM_BYTES, launch_y_2304},
    {2352, 14, 12, 14, YCfg<Rad<14, 12, 14>>::THREADS, YCfg<Rad<14, 12, 14>>::SMEM_BYTES, launch_y_2352},
    {2400, 16, 10, 15, YCfg<Rad<16, 10, 15>>::THREADS, YCfg<Rad<16, 10, 15>>::SMEM_BYTES, launch_y_2400},
    {2520, 15, 12, 14, YCfg<Rad<15, 12, 14>>::THREADS, YCfg<Rad<15, 12, 14>>::SMEM_BYTES, launch_y_2520},
    {2560, 16, 10, 16, YCfg<Rad<16, 10, 16>>::THREADS, YCfg<Rad<16, 10, 16>>::SMEM_BYTES, launch_y_2560},
    {2688, 16, 12, 14, YCfg<Rad<16, 12, 14>>::THREADS, YCfg<Rad<16, 12, 14>>::SMEM_BYTES, launch_y_2688},
    {2700, 15, 12, 15, YCfg<Rad<15, 12, 15>>::THREADS, YCfg<Rad<15, 12, 15>>::SMEM_BYTES, launch_y_2700},
    {2744, 14, 14, 14, YCfg<Rad<14, 14, 14>>::THREADS, YCfg<Rad<14, 14, 14>>::SMEM_BYTES, launch_y_2744},
    {2880, 16, 12, 15, YCfg<Rad<16, 12, 15>>::THREADS, YCfg<Rad<16, 12, 15>>::SMEM_BYTES, launch_y_2880},
    {2940, 15, 14, 14, YCfg<Rad<15, 14, 14>>::THREADS, YCfg<Rad<15, 14, 14>>::SMEM_BYTES, launch_y_2940},
    {3072, 16, 12, 16, YCfg<Rad<16, 12, 16>>::THREADS, YCfg<Rad<16, 12, 16>>::SMEM_BYTES, launch_y_3072},
    {3136, 16, 14, 14, YCfg<Rad<16, 14, 14>>::THREADS, YCfg<Rad<16, 14, 14>>::SMEM_BYTES, launch_y_3136},
    {3150, 15, 14, 15, YCfg<Rad<15, 14, 15>>::THREADS, YCfg<Rad<15, 14, 15>>::SMEM_BYTES, launch_y_3150},
};
}  // namespace dwcu
