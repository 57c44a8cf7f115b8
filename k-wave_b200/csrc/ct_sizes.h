// Transform lengths with compile-time FFT kernels: every 2^a 3^b 5^c length
// from 64 to 1024 (61 lengths).  build.py generates one translation
// unit per length (explicit instantiation of CtKernels<N>) and compiles them
// in parallel; any other length runs on the runtime-plan engine.
#pragma once

#define KWB_CT_SIZES(X) \
  X(64) X(72) X(75) X(80) X(81) X(90) X(96) X(100) X(108) X(120) X(125) X(128) X(135) X(144) X(150) \
  X(160) X(162) X(180) X(192) X(200) X(216) X(225) X(240) X(243) X(250) X(256) X(270) X(288) X(300) \
  X(320) X(324) X(360) X(375) X(384) X(400) X(405) X(432) X(450) X(480) X(486) X(500) X(512) X(540) \
  X(576) X(600) X(625) X(640) X(648) X(675) X(720) X(729) X(750) X(768) X(800) X(810) X(864) X(900) \
  X(960) X(972) X(1000) X(1024)
