// Line lengths with compiled mixed-radix kernels, in eight groups each (one translation unit
// per group, so they compile in parallel).  Conventional passes (PTX_MIX_GROUPk): every
// {2,3,5}-smooth length from 6 to 1000 that is not a power of two.  Fourier ptychography
// passes (PTX_MIXFPM_GROUPk): every {2,3,5}-smooth length from 4 to 1024, the powers of two
// included (an FPM problem takes them when another of its sides is not a power of two).
// Coded / near-field passes (PTX_MIXCODED_GROUPk): every {2,3,5}-smooth field side from 16 to
// 1000 that is not a power of two.
#pragma once

#define PTX_MIX_GROUP0(X) X(6) X(25) X(54) X(100) X(162) X(250) X(384) X(540) X(729) X(972)
#define PTX_MIX_GROUP1(X) X(9) X(27) X(60) X(108) X(180) X(270) X(400) X(576) X(750) X(1000)
#define PTX_MIX_GROUP2(X) X(10) X(30) X(72) X(120) X(192) X(288) X(405) X(600) X(768)
#define PTX_MIX_GROUP3(X) X(12) X(36) X(75) X(125) X(200) X(300) X(432) X(625) X(800)
#define PTX_MIX_GROUP4(X) X(15) X(40) X(80) X(135) X(216) X(320) X(450) X(640) X(810)
#define PTX_MIX_GROUP5(X) X(18) X(45) X(81) X(144) X(225) X(324) X(480) X(648) X(864)
#define PTX_MIX_GROUP6(X) X(20) X(48) X(90) X(150) X(240) X(360) X(486) X(675) X(900)
#define PTX_MIX_GROUP7(X) X(24) X(50) X(96) X(160) X(243) X(375) X(500) X(720) X(960)

#define PTX_MIXFPM_GROUP0(X) X(4) X(16) X(36) X(72) X(120) X(180) X(256) X(384) X(512) X(720) X(960)
#define PTX_MIXFPM_GROUP1(X) X(5) X(18) X(40) X(75) X(125) X(192) X(270) X(400) X(540) X(729) X(972)
#define PTX_MIXFPM_GROUP2(X) X(6) X(20) X(45) X(80) X(128) X(200) X(288) X(405) X(576) X(750) X(1000)
#define PTX_MIXFPM_GROUP3(X) X(8) X(24) X(48) X(81) X(135) X(216) X(300) X(432) X(600) X(768) X(1024)
#define PTX_MIXFPM_GROUP4(X) X(9) X(25) X(50) X(90) X(144) X(225) X(320) X(450) X(625) X(800)
#define PTX_MIXFPM_GROUP5(X) X(10) X(27) X(54) X(96) X(150) X(240) X(324) X(480) X(640) X(810)
#define PTX_MIXFPM_GROUP6(X) X(12) X(30) X(60) X(100) X(160) X(243) X(360) X(486) X(648) X(864)
#define PTX_MIXFPM_GROUP7(X) X(15) X(32) X(64) X(108) X(162) X(250) X(375) X(500) X(675) X(900)

#define PTX_MIXCODED_GROUP0(X) X(18) X(45) X(81) X(144) X(225) X(324) X(480) X(648) X(864)
#define PTX_MIXCODED_GROUP1(X) X(20) X(48) X(90) X(150) X(240) X(360) X(486) X(675) X(900)
#define PTX_MIXCODED_GROUP2(X) X(24) X(50) X(96) X(160) X(243) X(375) X(500) X(720) X(960)
#define PTX_MIXCODED_GROUP3(X) X(25) X(54) X(100) X(162) X(250) X(384) X(540) X(729) X(972)
#define PTX_MIXCODED_GROUP4(X) X(27) X(60) X(108) X(180) X(270) X(400) X(576) X(750) X(1000)
#define PTX_MIXCODED_GROUP5(X) X(30) X(72) X(120) X(192) X(288) X(405) X(600) X(768)
#define PTX_MIXCODED_GROUP6(X) X(36) X(75) X(125) X(200) X(300) X(432) X(625) X(800)
#define PTX_MIXCODED_GROUP7(X) X(40) X(80) X(135) X(216) X(320) X(450) X(640) X(810)
