// Transform lengths of the TMA-fed column passes (the y pass and the fused
// last-axis operator): every 2^a 3^b 5^c length from 64 to 256 (a tensor
// copy's box holds at most 256 elements along a dimension).  build.py
// generates one translation unit per length for the fused operator
// (fused_tma_N.cu, an explicit instantiation of fused_tma_cls<N>) and
// compiles them in parallel.
#pragma once

#define KWB_TMA_COL_SIZES(X)                                                                                   \
  X(64) X(72) X(75) X(80) X(81) X(90) X(96) X(100) X(108) X(120) X(125) X(128) X(135) X(144) X(150) X(160) \
  X(162) X(180) X(192) X(200) X(216) X(225) X(240) X(243) X(250) X(256)
