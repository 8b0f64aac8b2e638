// Generated by unicorn_b200/mech/codegen.py: the in-place species-update program
// (src/lib/solvesp.f:85-2806) for a tile whose RC block is held on chip.
// RC rows: 256 in tensor memory (row i in columns 2i, 2i+1: low and high
// word), 281 in shared memory. Requires RCS(i) (shared-memory row i of the
// cell), TM_LD(bank, q, col) (load the double at column col into slot q of a
// register bank), TM_WAIT(bank) (wait for the loads of that bank), RCT(bank, q),
// and the accessors of the in-place program (YO, YN, YOS, Y0, SOUR, WM, FACE_SUM,
// FACE_NBR, UC_UPDATE_TAIL; scalars rho, dt, sor1, sor2, rsd).
// 74 segments and 881 tensor-memory loads per cell and pass.
#pragma once
#define UC_TR_NT 256
#define UC_TR_NS 281
#define UC_TR_SEG 12
#define UC_TR_SHADOW_SAVE() do { YOS(0) = YO(2); YOS(1) = YO(4); YOS(2) = YO(6); YOS(3) = YO(13); YOS(4) = YO(16); YOS(5) = YO(14); YOS(6) = YO(8); YOS(7) = YO(22); } while (0)
#define UC_UPDATE_PROGRAM_TR() do { \
    double prod = 0.0, extra, loss, rhs1, rhs2, ppp, fnew; \
    TM_LD(0, 0, 6); \
    TM_LD(0, 1, 10); \
    TM_LD(0, 2, 16); \
    TM_LD(0, 3, 44); \
    TM_LD(0, 4, 68); \
    TM_LD(0, 5, 100); \
    TM_LD(0, 6, 128); \
    TM_LD(0, 7, 148); \
    TM_LD(0, 8, 168); \
    TM_LD(0, 9, 172); \
    TM_LD(0, 10, 200); \
    TM_LD(0, 11, 228); \
    TM_WAIT(0); \
    TM_LD(1, 0, 240); \
    TM_LD(1, 1, 244); \
    TM_LD(1, 2, 264); \
    TM_LD(1, 3, 288); \
    TM_LD(1, 4, 312); \
    TM_LD(1, 5, 332); \
    TM_LD(1, 6, 364); \
    TM_LD(1, 7, 368); \
    TM_LD(1, 8, 4); \
    TM_LD(1, 9, 8); \
    TM_LD(1, 10, 18); \
    TM_LD(1, 11, 46); \
    prod = ((YO(4) * YO(2)) * RCT(0, 0)); \
    prod = prod + ((YO(5) * YO(2)) * RCT(0, 1)); \
    prod = prod + ((YO(2) * YO(2)) * RCT(0, 2)); \
    prod = prod + ((YO(6) * YO(2)) * RCT(0, 3)); \
    prod = prod + ((YO(7) * YO(2)) * RCT(0, 4)); \
    prod = prod + ((YO(10) * YO(2)) * RCT(0, 5)); \
    prod = prod + ((YO(11) * YO(2)) * RCT(0, 6)); \
    prod = prod + ((YO(12) * YO(2)) * RCT(0, 7)); \
    prod = prod + ((YO(13) * YO(2)) * RCT(0, 8)); \
    prod = prod + ((YO(13) * YO(2)) * RCT(0, 9)); \
    prod = prod + ((YO(13) * YO(13)) * RCT(0, 10)); \
    prod = prod + ((YO(14) * YO(2)) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 70); \
    TM_LD(0, 1, 102); \
    TM_LD(0, 2, 130); \
    TM_LD(0, 3, 150); \
    TM_LD(0, 4, 170); \
    TM_LD(0, 5, 174); \
    TM_LD(0, 6, 202); \
    TM_LD(0, 7, 230); \
    TM_LD(0, 8, 242); \
    TM_LD(0, 9, 246); \
    TM_LD(0, 10, 266); \
    TM_LD(0, 11, 290); \
    prod = prod + ((YO(14) * YO(3)) * RCT(1, 0)); \
    prod = prod + ((YO(14) * YO(1)) * RCT(1, 1)); \
    prod = prod + ((YO(17) * YO(2)) * RCT(1, 2)); \
    prod = prod + ((YO(19) * YO(2)) * RCT(1, 3)); \
    prod = prod + ((YO(18) * YO(2)) * RCT(1, 4)); \
    prod = prod + ((YO(16) * YO(2)) * RCT(1, 5)); \
    prod = prod + (YO(16) * RCT(1, 6)); \
    prod = prod + ((YO(22) * YO(2)) * RCT(1, 7)); \
    prod = prod + ((YO(28) * YO(2)) * RCS(50)); \
    prod = prod + ((YO(29) * YO(2)) * RCS(64)); \
    prod = prod + ((YO(29) * YO(2)) * RCS(66)); \
    prod = prod + ((YO(23) * YO(2)) * RCS(76)); \
    prod = prod + ((YO(31) * YO(2)) * RCS(98)); \
    prod = prod + ((YO(31) * YO(2)) * RCS(100)); \
    prod = prod + ((YO(30) * YO(2)) * RCS(118)); \
    prod = prod + ((YO(30) * YO(2)) * RCS(120)); \
    prod = prod + ((YO(30) * YO(2)) * RCS(122)); \
    prod = prod + ((YO(38) * YO(2)) * RCS(178)); \
    prod = prod + ((YO(39) * YO(2)) * RCS(198)); \
    prod = prod + ((YO(40) * YO(2)) * RCS(212)); \
    prod = prod + ((YO(40) * YO(2)) * RCS(214)); \
    prod = prod + ((YO(43) * YO(2)) * RCS(236)); \
    prod = prod + ((YO(46) * YO(2)) * RCS(254)); \
    prod = prod + ((YO(48) * YO(2)) * RCS(263)); \
    prod = prod + ((YO(48) * YO(2)) * RCS(269)); \
    prod = prod + ((YO(48) * YO(2)) * RCS(271)); \
    prod = prod + ((YO(47) * YO(2)) * RCS(277)); \
    prod = prod + (SOUR(0) * YO(21)); \
    extra = (1.0 * ((YO(46) * YO(2)) * RCS(251))); \
    extra = extra + (1.0 * ((YO(46) * YO(2)) * RCS(252))); \
    extra = extra + (1.0 * ((YO(46) * YO(2)) * RCS(253))); \
    rhs1 = rho * Y0(0) + dt * WM(0) * (prod + extra); \
    loss = (YO(3) * RCT(1, 8)); \
    loss = loss + (YO(4) * RCT(1, 9)); \
    loss = loss + RCT(1, 10); \
    loss = loss + (YO(1) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 314); \
    TM_LD(1, 1, 334); \
    TM_LD(1, 2, 366); \
    TM_LD(1, 3, 370); \
    TM_LD(1, 4, 2); \
    TM_LD(1, 5, 24); \
    TM_LD(1, 6, 38); \
    TM_LD(1, 7, 44); \
    TM_LD(1, 8, 52); \
    TM_LD(1, 9, 56); \
    TM_LD(1, 10, 64); \
    TM_LD(1, 11, 94); \
    loss = loss + (YO(6) * RCT(0, 0)); \
    loss = loss + (YO(8) * RCT(0, 1)); \
    loss = loss + (YO(10) * RCT(0, 2)); \
    loss = loss + (YO(13) * RCT(0, 3)); \
    loss = loss + (YO(14) * RCT(0, 4)); \
    loss = loss + (YO(15) * RCT(0, 5)); \
    loss = loss + (YO(16) * RCT(0, 6)); \
    loss = loss + (YO(20) * RCT(0, 7)); \
    loss = loss + (YO(8) * RCT(0, 8)); \
    loss = loss + (YO(9) * RCT(0, 9)); \
    loss = loss + (YO(11) * RCT(0, 10)); \
    loss = loss + (YO(18) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 118); \
    TM_LD(0, 1, 142); \
    TM_LD(0, 2, 162); \
    TM_LD(0, 3, 194); \
    TM_LD(0, 4, 198); \
    TM_LD(0, 5, 246); \
    TM_LD(0, 6, 254); \
    TM_LD(0, 7, 282); \
    TM_LD(0, 8, 326); \
    TM_LD(0, 9, 354); \
    TM_LD(0, 10, 378); \
    TM_LD(0, 11, 382); \
    loss = loss + (YO(16) * RCT(1, 0)); \
    loss = loss + (YO(22) * RCT(1, 1)); \
    loss = loss + (YO(21) * RCT(1, 2)); \
    loss = loss + (YO(21) * RCT(1, 3)); \
    loss = loss + (YO(11) * RCS(51)); \
    loss = loss + (YO(28) * RCS(65)); \
    loss = loss + (YO(17) * RCS(67)); \
    loss = loss + (YO(25) * RCS(77)); \
    loss = loss + (YO(34) * RCS(99)); \
    loss = loss + (YO(23) * RCS(101)); \
    loss = loss + (YO(33) * RCS(119)); \
    loss = loss + (YO(32) * RCS(121)); \
    loss = loss + (YO(35) * RCS(123)); \
    loss = loss + (YO(36) * RCS(179)); \
    loss = loss + (YO(38) * RCS(199)); \
    loss = loss + (YO(41) * RCS(213)); \
    loss = loss + (YO(42) * RCS(215)); \
    loss = loss + ((YO(21) * YO(22)) * RCS(237)); \
    loss = loss + ((YO(48) * YO(18)) * RCS(255)); \
    loss = loss + ((YO(39) * YO(22)) * RCS(264)); \
    loss = loss + ((YO(16) * YO(38)) * RCS(270)); \
    loss = loss + ((YO(43) * YO(13)) * RCS(272)); \
    loss = loss + ((YO(22) * YO(16)) * RCS(278)); \
    rhs2 = -(dt * WM(0) * loss); \
    ppp = rho - FACE_SUM(0); \
    fnew = sor2 * YO(0) + (rhs1 - FACE_NBR(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(0) - fnew); \
    UC_UPDATE_TAIL(0); \
    prod = ((YO(4) * YO(3)) * RCT(1, 4)); \
    prod = prod + ((YO(3) * YO(3)) * RCT(1, 5)); \
    prod = prod + (YO(6) * RCT(1, 6)); \
    prod = prod + ((YO(6) * YO(2)) * RCT(1, 7)); \
    prod = prod + ((YO(6) * YO(3)) * RCT(1, 8)); \
    prod = prod + ((YO(6) * YO(4)) * RCT(1, 9)); \
    prod = prod + ((YO(6) * YO(6)) * RCT(1, 10)); \
    prod = prod + ((YO(9) * YO(3)) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 0); \
    TM_LD(1, 1, 26); \
    TM_LD(1, 2, 36); \
    TM_LD(1, 3, 46); \
    TM_LD(1, 4, 54); \
    TM_LD(1, 5, 58); \
    TM_LD(1, 6, 66); \
    TM_LD(1, 7, 92); \
    TM_LD(1, 8, 116); \
    TM_LD(1, 9, 140); \
    TM_LD(1, 10, 160); \
    TM_LD(1, 11, 192); \
    prod = prod + ((YO(8) * YO(6)) * RCT(0, 0)); \
    prod = prod + ((YO(10) * YO(6)) * RCT(0, 1)); \
    prod = prod + ((YO(13) * YO(6)) * RCT(0, 2)); \
    prod = prod + ((YO(11) * YO(4)) * RCT(0, 3)); \
    prod = prod + ((YO(17) * YO(3)) * RCT(0, 4)); \
    prod = prod + (((YO(8) * YO(4)) * YO(2)) * RCS(1)); \
    prod = prod + (YN(0) * (YO(9) * RCT(0, 5))); \
    prod = prod + (((YO(8) * YO(4)) * YO(2)) * RCS(5)); \
    prod = prod + ((YO(10) * YO(3)) * RCT(0, 6)); \
    prod = prod + ((YO(11) * YO(6)) * RCT(0, 7)); \
    prod = prod + ((YO(16) * YO(6)) * RCT(0, 8)); \
    prod = prod + ((YO(22) * YO(6)) * RCT(0, 9)); \
    prod = prod + ((YO(11) * YO(10)) * RCT(0, 10)); \
    prod = prod + ((YO(23) * YO(3)) * RCT(0, 11)); \
    prod = prod + ((YO(21) * YO(6)) * RCS(11)); \
    prod = prod + ((YO(11) * YO(8)) * RCS(17)); \
    prod = prod + (((YO(8) * YO(8)) * YO(4)) * RCS(37)); \
    prod = prod + (((YO(9) * YO(8)) * YO(2)) * RCS(39)); \
    prod = prod + ((YO(26) * YO(3)) * RCS(45)); \
    prod = prod + ((YO(20) * YO(9)) * RCS(47)); \
    prod = prod + ((YO(10) * YO(8)) * RCS(49)); \
    prod = prod + ((YO(11) * YO(6)) * RCS(57)); \
    prod = prod + ((YO(28) * YO(6)) * RCS(73)); \
    prod = prod + (((YO(11) * YO(8)) * YO(4)) * RCS(83)); \
    prod = prod + ((YO(23) * YO(6)) * RCS(88)); \
    prod = prod + ((YO(34) * YO(6)) * RCS(111)); \
    prod = prod + ((YO(31) * YO(6)) * RCS(145)); \
    prod = prod + ((YO(31) * YO(6)) * RCS(155)); \
    prod = prod + ((YO(37) * YO(6)) * RCS(172)); \
    prod = prod + ((YO(25) * YO(10)) * RCS(177)); \
    prod = prod + ((YO(36) * YO(6)) * RCS(181)); \
    prod = prod + (((YO(13) * YO(10)) * YO(8)) * RCS(191)); \
    prod = prod + ((YO(38) * YO(6)) * RCS(200)); \
    prod = prod + ((YO(41) * YO(6)) * RCS(209)); \
    prod = prod + ((YO(42) * YO(6)) * RCS(211)); \
    prod = prod + ((YO(39) * YO(6)) * RCS(229)); \
    prod = prod + ((YO(39) * YO(6)) * RCS(231)); \
    prod = prod + (((YO(21) * YO(38)) * YO(6)) * RCS(243)); \
    prod = prod + (((YO(22) * YO(36)) * YO(6)) * RCS(245)); \
    extra = 0.0; \
    rhs1 = rho * Y0(1) + dt * WM(1) * (prod + extra); \
    TM_WAIT(1); \
    TM_LD(0, 0, 196); \
    TM_LD(0, 1, 244); \
    TM_LD(0, 2, 252); \
    TM_LD(0, 3, 280); \
    TM_LD(0, 4, 324); \
    TM_LD(0, 5, 352); \
    TM_LD(0, 6, 376); \
    TM_LD(0, 7, 380); \
    TM_LD(0, 8, 2); \
    TM_LD(0, 9, 4); \
    TM_LD(0, 10, 8); \
    TM_LD(0, 11, 18); \
    loss = (YO(2) * RCT(1, 0)); \
    loss = loss + RCT(1, 1); \
    loss = loss + (YO(2) * RCT(1, 2)); \
    loss = loss + (YN(0) * RCT(1, 3)); \
    loss = loss + (YO(4) * RCT(1, 4)); \
    loss = loss + (YO(5) * RCT(1, 5)); \
    loss = loss + (YO(7) * RCT(1, 6)); \
    loss = loss + (YO(8) * RCT(1, 7)); \
    loss = loss + (YO(10) * RCT(1, 8)); \
    loss = loss + (YO(11) * RCT(1, 9)); \
    loss = loss + (YO(12) * RCT(1, 10)); \
    loss = loss + (YO(13) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 22); \
    TM_LD(1, 1, 30); \
    TM_LD(1, 2, 38); \
    TM_LD(1, 3, 42); \
    TM_LD(1, 4, 46); \
    TM_LD(1, 5, 50); \
    TM_LD(1, 6, 70); \
    TM_LD(1, 7, 74); \
    TM_LD(1, 8, 84); \
    TM_LD(1, 9, 96); \
    TM_LD(1, 10, 102); \
    TM_LD(1, 11, 108); \
    loss = loss + (YO(13) * RCT(0, 0)); \
    loss = loss + (YO(15) * RCS(0)); \
    loss = loss + (YO(14) * RCT(0, 1)); \
    loss = loss + (YO(14) * RCS(4)); \
    loss = loss + (YO(20) * RCT(0, 2)); \
    loss = loss + (YO(17) * RCT(0, 3)); \
    loss = loss + (YO(18) * RCT(0, 4)); \
    loss = loss + (YO(16) * RCT(0, 5)); \
    loss = loss + (YO(22) * RCT(0, 6)); \
    loss = loss + (YO(22) * RCT(0, 7)); \
    loss = loss + (YO(22) * RCS(10)); \
    loss = loss + (YO(21) * RCS(16)); \
    loss = loss + (YO(26) * RCS(36)); \
    loss = loss + (YO(26) * RCS(38)); \
    loss = loss + (YO(27) * RCS(44)); \
    loss = loss + (YO(27) * RCS(46)); \
    loss = loss + (YO(27) * RCS(48)); \
    loss = loss + (YO(28) * RCS(56)); \
    loss = loss + (YO(29) * RCS(72)); \
    loss = loss + (YO(23) * RCS(82)); \
    loss = loss + (YO(31) * RCS(89)); \
    loss = loss + (YO(31) * RCS(110)); \
    loss = loss + (YO(35) * RCS(144)); \
    loss = loss + (YO(32) * RCS(154)); \
    loss = loss + (YO(36) * RCS(173)); \
    loss = loss + (YO(37) * RCS(176)); \
    loss = loss + (YO(38) * RCS(180)); \
    loss = loss + (YO(36) * RCS(190)); \
    loss = loss + (YO(39) * RCS(201)); \
    loss = loss + (YO(40) * RCS(208)); \
    loss = loss + (YO(40) * RCS(210)); \
    loss = loss + (YO(41) * RCS(228)); \
    loss = loss + (YO(42) * RCS(230)); \
    loss = loss + (YO(45) * RCS(242)); \
    loss = loss + (YO(45) * RCS(244)); \
    loss = loss + (0.5 * SOUR(2)); \
    rhs2 = -(dt * WM(1) * loss); \
    ppp = rho - FACE_SUM(1); \
    fnew = sor2 * YO(1) + (rhs1 - FACE_NBR(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(1) - fnew); \
    UC_UPDATE_TAIL(1); \
    prod = ((YO(4) * YO(3)) * RCT(0, 8)); \
    prod = prod + (YN(0) * (YO(3) * RCT(0, 9))); \
    prod = prod + (YN(0) * (YO(4) * RCT(0, 10))); \
    prod = prod + (YN(0) * RCT(0, 11)); \
    prod = prod + (YN(0) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 126); \
    TM_LD(0, 1, 130); \
    TM_LD(0, 2, 150); \
    TM_LD(0, 3, 170); \
    TM_LD(0, 4, 174); \
    TM_LD(0, 5, 180); \
    TM_LD(0, 6, 184); \
    TM_LD(0, 7, 204); \
    TM_LD(0, 8, 210); \
    TM_LD(0, 9, 216); \
    TM_LD(0, 10, 230); \
    TM_LD(0, 11, 232); \
    prod = prod + (YO(5) * RCT(1, 0)); \
    prod = prod + (YO(4) * RCT(1, 1)); \
    prod = prod + (YO(6) * RCT(1, 2)); \
    prod = prod + ((YO(4) * YO(4)) * RCT(1, 3)); \
    prod = prod + (YN(1) * (YN(0) * RCT(1, 4))); \
    prod = prod + ((YO(5) * YO(3)) * RCT(1, 5)); \
    prod = prod + (YN(0) * (YO(6) * RCT(1, 6))); \
    prod = prod + ((YO(5) * YO(4)) * RCT(1, 7)); \
    prod = prod + ((YO(8) * YO(4)) * RCT(1, 8)); \
    prod = prod + (YO(10) * RCT(1, 9)); \
    prod = prod + (YN(0) * (YO(8) * RCT(1, 10))); \
    prod = prod + ((YO(10) * YO(3)) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 248); \
    TM_LD(1, 1, 256); \
    TM_LD(1, 2, 266); \
    TM_LD(1, 3, 270); \
    TM_LD(1, 4, 284); \
    TM_LD(1, 5, 290); \
    TM_LD(1, 6, 304); \
    TM_LD(1, 7, 314); \
    TM_LD(1, 8, 328); \
    TM_LD(1, 9, 334); \
    TM_LD(1, 10, 344); \
    TM_LD(1, 11, 360); \
    prod = prod + (YO(11) * RCT(0, 0)); \
    prod = prod + (YN(0) * (YO(10) * RCT(0, 1))); \
    prod = prod + (YN(0) * (YO(13) * RCT(0, 2))); \
    prod = prod + (YN(0) * (YO(14) * RCT(0, 3))); \
    prod = prod + (YN(0) * (YO(15) * RCT(0, 4))); \
    prod = prod + ((YO(13) * YO(3)) * RCT(0, 5)); \
    prod = prod + ((YO(13) * YO(14)) * RCT(0, 6)); \
    prod = prod + ((YO(13) * YO(13)) * RCT(0, 7)); \
    prod = prod + (YO(12) * RCT(0, 8)); \
    prod = prod + ((YO(15) * YO(4)) * RCT(0, 9)); \
    prod = prod + (YN(1) * (YO(15) * RCS(0))); \
    prod = prod + (YN(0) * (YO(20) * RCT(0, 10))); \
    prod = prod + ((YO(14) * YO(4)) * RCT(0, 11)); \
    prod = prod + ((YO(14) * YO(3)) * RCS(2)); \
    prod = prod + ((YO(14) * YO(3)) * RCS(2)); \
    prod = prod + (YN(1) * (YO(14) * RCS(4))); \
    prod = prod + ((YO(14) * YO(14)) * RCS(6)); \
    prod = prod + ((YO(14) * YO(14)) * RCS(6)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 370); \
    TM_LD(0, 1, 372); \
    TM_LD(0, 2, 384); \
    TM_LD(0, 3, 396); \
    TM_LD(0, 4, 424); \
    TM_LD(0, 5, 432); \
    TM_LD(0, 6, 438); \
    TM_LD(0, 7, 442); \
    TM_LD(0, 8, 450); \
    TM_LD(0, 9, 466); \
    TM_LD(0, 10, 474); \
    TM_LD(0, 11, 0); \
    prod = prod + ((YO(20) * YO(3)) * RCT(1, 0)); \
    prod = prod + ((YO(20) * YO(5)) * RCT(1, 1)); \
    prod = prod + (YN(0) * (YO(11) * RCT(1, 2))); \
    prod = prod + ((YO(15) * YO(5)) * RCT(1, 3)); \
    prod = prod + (YO(17) * RCT(1, 4)); \
    prod = prod + (YN(0) * (YO(18) * RCT(1, 5))); \
    prod = prod + (YO(19) * RCT(1, 6)); \
    prod = prod + (YN(0) * (YO(16) * RCT(1, 7))); \
    prod = prod + (YO(18) * RCT(1, 8)); \
    prod = prod + (YN(0) * (YO(22) * RCT(1, 9))); \
    prod = prod + ((YO(16) * YO(3)) * RCT(1, 10)); \
    prod = prod + (YO(16) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 6); \
    TM_LD(1, 1, 10); \
    TM_LD(1, 2, 16); \
    TM_LD(1, 3, 20); \
    TM_LD(1, 4, 28); \
    TM_LD(1, 5, 36); \
    TM_LD(1, 6, 40); \
    TM_LD(1, 7, 44); \
    TM_LD(1, 8, 48); \
    TM_LD(1, 9, 68); \
    TM_LD(1, 10, 72); \
    TM_LD(1, 11, 86); \
    prod = prod + (YN(0) * (YO(21) * RCT(0, 0))); \
    prod = prod + (YO(22) * RCT(0, 1)); \
    prod = prod + ((YO(21) * YO(3)) * RCS(12)); \
    prod = prod + ((YO(21) * YO(4)) * RCS(18)); \
    prod = prod + ((YO(13) * YO(8)) * RCS(23)); \
    prod = prod + ((YO(15) * YO(8)) * RCS(31)); \
    prod = prod + ((YO(26) * YO(4)) * RCS(32)); \
    prod = prod + ((YO(26) * YO(3)) * RCS(34)); \
    prod = prod + (YN(1) * (YO(26) * RCS(38))); \
    prod = prod + ((YO(27) * YO(4)) * RCS(40)); \
    prod = prod + (YN(0) * (YO(11) * RCS(51))); \
    prod = prod + ((YO(13) * YO(4)) * RCS(53)); \
    prod = prod + (YO(28) * RCT(0, 2)); \
    prod = prod + (YN(0) * (YO(28) * RCS(65))); \
    prod = prod + (YN(0) * (YO(17) * RCS(67))); \
    prod = prod + (YO(23) * RCT(0, 3)); \
    prod = prod + ((YO(13) * YO(10)) * RCS(75)); \
    prod = prod + (YN(0) * (YO(25) * RCS(77))); \
    prod = prod + ((YO(23) * YO(13)) * RCS(84)); \
    prod = prod + (YN(0) * (YO(34) * RCS(99))); \
    prod = prod + (YN(0) * (YO(23) * RCS(101))); \
    prod = prod + (YN(0) * (YO(33) * RCS(119))); \
    prod = prod + (YN(0) * (YO(32) * RCS(121))); \
    prod = prod + (YN(0) * (YO(35) * RCS(123))); \
    prod = prod + (YO(35) * RCT(0, 4)); \
    prod = prod + ((YO(13) * YO(28)) * RCS(149)); \
    prod = prod + ((YO(16) * YO(5)) * RCS(151)); \
    prod = prod + ((YO(16) * YO(5)) * RCS(159)); \
    prod = prod + ((YO(13) * YO(28)) * RCS(161)); \
    prod = prod + (YO(32) * RCT(0, 5)); \
    prod = prod + ((YO(13) * YO(21)) * RCS(168)); \
    prod = prod + (YO(36) * RCT(0, 6)); \
    prod = prod + (YO(38) * RCT(0, 7)); \
    prod = prod + (YN(0) * (YO(36) * RCS(179))); \
    prod = prod + ((YO(39) * YO(3)) * RCS(196)); \
    prod = prod + (YN(0) * (YO(38) * RCS(199))); \
    prod = prod + (YO(39) * RCT(0, 8)); \
    prod = prod + ((YO(16) * YO(13)) * RCS(205)); \
    prod = prod + ((YO(13) * YO(22)) * RCS(206)); \
    prod = prod + (YN(0) * (YO(41) * RCS(213))); \
    prod = prod + (YN(0) * (YO(42) * RCS(215))); \
    prod = prod + (YO(41) * RCT(0, 9)); \
    prod = prod + (YO(42) * RCT(0, 10)); \
    prod = prod + (YO(43) * RCS(232)); \
    prod = prod + ((YO(22) * YO(16)) * RCS(235)); \
    prod = prod + (YN(0) * ((YO(21) * YO(22)) * RCS(237))); \
    prod = prod + ((YO(43) * YO(4)) * RCS(238)); \
    prod = prod + 0.0; \
    prod = prod + 0.0; \
    prod = prod + 0.0; \
    prod = prod + (YN(0) * ((YO(48) * YO(18)) * RCS(255))); \
    prod = prod + (YN(0) * ((YO(39) * YO(22)) * RCS(264))); \
    prod = prod + (((YO(16) * YO(16)) * YO(13)) * RCS(266)); \
    prod = prod + ((YO(39) * YO(18)) * RCS(268)); \
    prod = prod + (YN(0) * ((YO(16) * YO(38)) * RCS(270))); \
    prod = prod + (YN(0) * ((YO(43) * YO(13)) * RCS(272))); \
    prod = prod + ((YO(16) * YO(18)) * RCS(274)); \
    prod = prod + ((YO(39) * YO(13)) * RCS(276)); \
    prod = prod + (YN(0) * ((YO(22) * YO(16)) * RCS(278))); \
    prod = prod + ((YO(47) * YO(4)) * RCS(279)); \
    prod = prod + (SOUR(3) * YO(4)); \
    extra = 0.0; \
    rhs1 = rho * Y0(2) + dt * WM(2) * (prod + extra); \
    loss = (YN(1) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 98); \
    TM_LD(0, 1, 100); \
    TM_LD(0, 2, 110); \
    TM_LD(0, 3, 124); \
    TM_LD(0, 4, 128); \
    TM_LD(0, 5, 148); \
    TM_LD(0, 6, 168); \
    TM_LD(0, 7, 172); \
    TM_LD(0, 8, 182); \
    TM_LD(0, 9, 186); \
    TM_LD(0, 10, 206); \
    TM_LD(0, 11, 208); \
    loss = loss + (YO(4) * RCT(1, 0)); \
    loss = loss + (YO(5) * RCT(1, 1)); \
    loss = loss + (YO(2) * RCT(1, 2)); \
    loss = loss + (YO(2) * RCT(1, 2)); \
    loss = loss + (YO(4) * RCT(1, 3)); \
    loss = loss + (YO(3) * RCT(1, 4)); \
    loss = loss + (YN(1) * RCT(1, 5)); \
    loss = loss + (YO(6) * RCT(1, 6)); \
    loss = loss + (YO(6) * RCT(1, 7)); \
    loss = loss + (YO(6) * RCT(1, 8)); \
    loss = loss + (YO(7) * RCT(1, 9)); \
    loss = loss + (YO(7) * RCT(1, 10)); \
    loss = loss + (YO(9) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 218); \
    TM_LD(1, 1, 228); \
    TM_LD(1, 2, 234); \
    TM_LD(1, 3, 250); \
    TM_LD(1, 4, 258); \
    TM_LD(1, 5, 264); \
    TM_LD(1, 6, 268); \
    TM_LD(1, 7, 286); \
    TM_LD(1, 8, 288); \
    TM_LD(1, 9, 306); \
    TM_LD(1, 10, 312); \
    TM_LD(1, 11, 330); \
    loss = loss + (YO(8) * RCT(0, 0)); \
    loss = loss + (YO(10) * RCT(0, 1)); \
    loss = loss + (YO(9) * RCT(0, 2)); \
    loss = loss + (YO(10) * RCT(0, 3)); \
    loss = loss + (YO(11) * RCT(0, 4)); \
    loss = loss + (YO(12) * RCT(0, 5)); \
    loss = loss + (YO(13) * RCT(0, 6)); \
    loss = loss + (YO(13) * RCT(0, 7)); \
    loss = loss + (YO(11) * RCT(0, 8)); \
    loss = loss + (YO(16) * RCT(0, 9)); \
    loss = loss + (YO(18) * RCT(0, 10)); \
    loss = loss + (YO(13) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 332); \
    TM_LD(0, 1, 346); \
    TM_LD(0, 2, 362); \
    TM_LD(0, 3, 368); \
    TM_LD(0, 4, 374); \
    TM_LD(0, 5, 386); \
    TM_LD(0, 6, 398); \
    TM_LD(0, 7, 426); \
    TM_LD(0, 8, 434); \
    TM_LD(0, 9, 436); \
    TM_LD(0, 10, 440); \
    TM_LD(0, 11, 448); \
    loss = loss + (YO(11) * RCT(1, 0)); \
    loss = loss + ((YO(8) * YO(4)) * RCS(1)); \
    loss = loss + (YO(14) * RCT(1, 1)); \
    loss = loss + (YO(11) * RCT(1, 2)); \
    loss = loss + ((YO(8) * YO(2)) * RCS(3)); \
    loss = loss + ((YO(8) * YO(2)) * RCS(3)); \
    loss = loss + ((YO(8) * YO(4)) * RCS(5)); \
    loss = loss + ((YO(21) * YO(2)) * RCS(7)); \
    loss = loss + ((YO(21) * YO(2)) * RCS(7)); \
    loss = loss + (YO(8) * RCT(1, 3)); \
    loss = loss + (YO(11) * RCT(1, 4)); \
    loss = loss + (YO(17) * RCT(1, 5)); \
    loss = loss + (YO(17) * RCT(1, 6)); \
    loss = loss + (YO(11) * RCT(1, 7)); \
    loss = loss + (YO(19) * RCT(1, 8)); \
    loss = loss + (YO(18) * RCT(1, 9)); \
    loss = loss + (YO(18) * RCT(1, 10)); \
    loss = loss + (YO(16) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 464); \
    TM_LD(1, 1, 472); \
    TM_LD(1, 2, 0); \
    TM_LD(1, 3, 6); \
    TM_LD(1, 4, 14); \
    TM_LD(1, 5, 26); \
    TM_LD(1, 6, 30); \
    TM_LD(1, 7, 34); \
    TM_LD(1, 8, 48); \
    TM_LD(1, 9, 54); \
    TM_LD(1, 10, 82); \
    TM_LD(1, 11, 92); \
    loss = loss + (YO(16) * RCT(0, 0)); \
    loss = loss + (YO(23) * RCT(0, 1)); \
    loss = loss + (YO(22) * RCT(0, 2)); \
    loss = loss + (YO(22) * RCT(0, 3)); \
    loss = loss + (YO(21) * RCT(0, 4)); \
    loss = loss + (YO(26) * RCS(13)); \
    loss = loss + (YO(25) * RCS(19)); \
    loss = loss + (YO(25) * RCS(22)); \
    loss = loss + (YO(26) * RCS(30)); \
    loss = loss + ((YO(10) * YO(8)) * RCS(33)); \
    loss = loss + ((YO(8) * YO(8)) * RCS(35)); \
    loss = loss + ((YO(9) * YO(8)) * RCS(39)); \
    loss = loss + (YO(26) * RCS(41)); \
    loss = loss + (YO(28) * RCS(50)); \
    loss = loss + (YO(28) * RCS(52)); \
    loss = loss + (YO(11) * RCT(0, 5)); \
    loss = loss + (YO(29) * RCS(64)); \
    loss = loss + (YO(29) * RCS(66)); \
    loss = loss + (YO(25) * RCT(0, 6)); \
    loss = loss + (YO(23) * RCS(74)); \
    loss = loss + (YO(23) * RCS(76)); \
    loss = loss + ((YO(18) * YO(8)) * RCS(85)); \
    loss = loss + (YO(31) * RCS(98)); \
    loss = loss + (YO(31) * RCS(100)); \
    loss = loss + (YO(30) * RCS(118)); \
    loss = loss + (YO(30) * RCS(120)); \
    loss = loss + (YO(30) * RCS(122)); \
    loss = loss + (YO(31) * RCT(0, 7)); \
    loss = loss + (YO(35) * RCS(148)); \
    loss = loss + (YO(35) * RCS(150)); \
    loss = loss + (YO(32) * RCS(158)); \
    loss = loss + (YO(32) * RCS(160)); \
    loss = loss + (YO(31) * RCT(0, 8)); \
    loss = loss + (YO(36) * RCS(169)); \
    loss = loss + (YO(37) * RCT(0, 9)); \
    loss = loss + (YO(36) * RCT(0, 10)); \
    loss = loss + (YO(38) * RCS(178)); \
    loss = loss + ((YO(25) * YO(13)) * RCS(197)); \
    loss = loss + (YO(39) * RCS(198)); \
    loss = loss + (YO(38) * RCT(0, 11)); \
    loss = loss + (YO(39) * RCS(204)); \
    loss = loss + (YO(38) * RCS(207)); \
    loss = loss + (YO(40) * RCS(212)); \
    loss = loss + (YO(40) * RCS(214)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 106); \
    TM_LD(0, 1, 110); \
    TM_LD(0, 2, 134); \
    TM_LD(0, 3, 158); \
    TM_LD(0, 4, 182); \
    TM_LD(0, 5, 196); \
    TM_LD(0, 6, 242); \
    TM_LD(0, 7, 250); \
    TM_LD(0, 8, 252); \
    TM_LD(0, 9, 278); \
    TM_LD(0, 10, 294); \
    TM_LD(0, 11, 318); \
    loss = loss + (YO(39) * RCT(1, 0)); \
    loss = loss + (YO(39) * RCT(1, 1)); \
    loss = loss + ((YO(21) * YO(22)) * RCS(233)); \
    loss = loss + (YO(43) * RCS(234)); \
    loss = loss + (YO(43) * RCS(236)); \
    loss = loss + ((YO(44) * YO(38)) * RCS(239)); \
    loss = loss + (YO(46) * RCS(251)); \
    loss = loss + (YO(46) * RCS(252)); \
    loss = loss + (YO(46) * RCS(253)); \
    loss = loss + (YO(46) * RCS(254)); \
    loss = loss + (YO(48) * RCS(263)); \
    loss = loss + (YO(48) * RCS(265)); \
    loss = loss + (YO(48) * RCS(267)); \
    loss = loss + (YO(48) * RCS(269)); \
    loss = loss + (YO(48) * RCS(271)); \
    loss = loss + (YO(47) * RCS(273)); \
    loss = loss + (YO(47) * RCS(275)); \
    loss = loss + (YO(47) * RCS(277)); \
    loss = loss + ((YO(5) * YO(43)) * RCS(280)); \
    rhs2 = -(dt * WM(2) * loss); \
    ppp = rho - FACE_SUM(2); \
    fnew = sor2 * YO(2) + (rhs1 - FACE_NBR(2)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(2) - fnew); \
    UC_UPDATE_TAIL(2); \
    prod = (YN(2) * (YN(1) * RCT(1, 2))); \
    prod = prod + (YN(2) * (YO(4) * RCT(1, 3))); \
    prod = prod + ((YO(4) * YO(4)) * RCT(1, 4)); \
    prod = prod + (YN(1) * RCT(1, 5)); \
    prod = prod + (YN(1) * RCT(1, 5)); \
    prod = prod + (YO(4) * RCT(1, 6)); \
    prod = prod + (YO(6) * RCT(1, 7)); \
    prod = prod + (YN(2) * (YO(6) * RCT(1, 8))); \
    prod = prod + (YN(1) * (YO(4) * RCT(1, 9))); \
    prod = prod + ((YO(6) * YO(4)) * RCT(1, 10)); \
    prod = prod + (YN(1) * (YO(8) * RCT(1, 11))); \
    TM_WAIT(0); \
    TM_LD(1, 0, 322); \
    TM_LD(1, 1, 342); \
    TM_LD(1, 2, 346); \
    TM_LD(1, 3, 380); \
    TM_LD(1, 4, 2); \
    TM_LD(1, 5, 4); \
    TM_LD(1, 6, 12); \
    TM_LD(1, 7, 24); \
    TM_LD(1, 8, 28); \
    TM_LD(1, 9, 32); \
    TM_LD(1, 10, 50); \
    TM_LD(1, 11, 52); \
    prod = prod + ((YO(8) * YO(4)) * RCT(0, 0)); \
    prod = prod + (YN(2) * (YO(9) * RCT(0, 1))); \
    prod = prod + ((YO(10) * YO(4)) * RCT(0, 2)); \
    prod = prod + ((YO(13) * YO(4)) * RCT(0, 3)); \
    prod = prod + (YN(2) * (YO(11) * RCT(0, 4))); \
    prod = prod + (YN(1) * (YO(13) * RCT(0, 5))); \
    prod = prod + (YN(2) * ((YO(8) * YOS(0)) * RCS(3))); \
    prod = prod + (YN(0) * (YO(8) * RCT(0, 6))); \
    prod = prod + (YN(2) * (YO(8) * RCT(0, 7))); \
    prod = prod + (YN(1) * (YO(20) * RCT(0, 8))); \
    prod = prod + ((YO(4) * YO(11)) * RCT(0, 9)); \
    prod = prod + ((YO(18) * YO(4)) * RCT(0, 10)); \
    prod = prod + ((YO(16) * YO(4)) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 80); \
    TM_LD(0, 1, 94); \
    TM_LD(0, 2, 104); \
    TM_LD(0, 3, 108); \
    TM_LD(0, 4, 132); \
    TM_LD(0, 5, 156); \
    TM_LD(0, 6, 180); \
    TM_LD(0, 7, 198); \
    TM_LD(0, 8, 240); \
    TM_LD(0, 9, 248); \
    TM_LD(0, 10, 254); \
    TM_LD(0, 11, 276); \
    prod = prod + ((YO(13) * YO(11)) * RCT(1, 0)); \
    prod = prod + ((YO(13) * YO(10)) * RCT(1, 1)); \
    prod = prod + (YN(2) * (YO(23) * RCT(1, 2))); \
    prod = prod + (YN(1) * (YO(22) * RCT(1, 3))); \
    prod = prod + (YN(2) * (YO(26) * RCS(13))); \
    prod = prod + ((YO(14) * YO(8)) * RCS(15)); \
    prod = prod + ((YO(14) * YO(9)) * RCS(25)); \
    prod = prod + ((YO(26) * YO(4)) * RCS(27)); \
    prod = prod + (YN(2) * ((YO(8) * YO(8)) * RCS(35))); \
    prod = prod + ((YO(8) * YO(20)) * RCS(43)); \
    prod = prod + (YN(1) * (YO(27) * RCS(44))); \
    prod = prod + ((YO(28) * YO(4)) * RCS(69)); \
    prod = prod + ((YO(11) * YO(10)) * RCS(79)); \
    prod = prod + ((YO(34) * YO(4)) * RCS(95)); \
    prod = prod + ((YO(23) * YO(4)) * RCS(97)); \
    prod = prod + ((YO(33) * YO(4)) * RCS(125)); \
    prod = prod + ((YO(32) * YO(4)) * RCS(127)); \
    prod = prod + ((YO(35) * YO(4)) * RCS(129)); \
    prod = prod + ((YO(31) * YO(4)) * RCS(157)); \
    prod = prod + ((YO(16) * YO(8)) * RCS(167)); \
    prod = prod + ((YO(26) * YO(13)) * RCS(171)); \
    prod = prod + ((YO(18) * YO(10)) * RCS(193)); \
    prod = prod + (YN(2) * ((YO(25) * YO(13)) * RCS(197))); \
    prod = prod + ((YO(41) * YO(4)) * RCS(217)); \
    prod = prod + ((YO(42) * YO(4)) * RCS(219)); \
    extra = 0.0; \
    rhs1 = rho * Y0(3) + dt * WM(3) * (prod + extra); \
    loss = (YO(4) * RCT(1, 4)); \
    loss = loss + (YN(0) * RCT(1, 5)); \
    loss = loss + (YO(5) * RCT(1, 6)); \
    loss = loss + (YO(3) * RCT(1, 7)); \
    loss = loss + (YO(3) * RCT(1, 7)); \
    loss = loss + (YN(2) * RCT(1, 8)); \
    loss = loss + (YO(4) * RCT(1, 9)); \
    loss = loss + (YO(5) * RCT(1, 10)); \
    loss = loss + (YO(6) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 292); \
    TM_LD(1, 1, 316); \
    TM_LD(1, 2, 320); \
    TM_LD(1, 3, 340); \
    TM_LD(1, 4, 344); \
    TM_LD(1, 5, 382); \
    TM_LD(1, 6, 0); \
    TM_LD(1, 7, 4); \
    TM_LD(1, 8, 10); \
    TM_LD(1, 9, 12); \
    TM_LD(1, 10, 22); \
    TM_LD(1, 11, 28); \
    loss = loss + (YO(7) * RCT(0, 0)); \
    loss = loss + (YO(9) * RCT(0, 1)); \
    loss = loss + (YO(10) * RCT(0, 2)); \
    loss = loss + (YO(10) * RCT(0, 3)); \
    loss = loss + (YO(11) * RCT(0, 4)); \
    loss = loss + (YO(12) * RCT(0, 5)); \
    loss = loss + (YO(13) * RCT(0, 6)); \
    loss = loss + (YO(17) * RCT(0, 7)); \
    loss = loss + (YO(14) * RCS(2)); \
    loss = loss + (YO(14) * RCT(0, 8)); \
    loss = loss + (YO(20) * RCT(0, 9)); \
    loss = loss + (YO(10) * RCT(0, 10)); \
    loss = loss + (YO(17) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 34); \
    TM_LD(0, 1, 40); \
    TM_LD(0, 2, 52); \
    TM_LD(0, 3, 58); \
    TM_LD(0, 4, 62); \
    TM_LD(0, 5, 72); \
    TM_LD(0, 6, 78); \
    TM_LD(0, 7, 80); \
    TM_LD(0, 8, 86); \
    TM_LD(0, 9, 88); \
    TM_LD(0, 10, 104); \
    TM_LD(0, 11, 114); \
    loss = loss + (YO(19) * RCT(1, 0)); \
    loss = loss + (YO(18) * RCT(1, 1)); \
    loss = loss + (YO(18) * RCT(1, 2)); \
    loss = loss + (YO(16) * RCT(1, 3)); \
    loss = loss + (YO(16) * RCT(1, 4)); \
    loss = loss + (YO(23) * RCT(1, 5)); \
    loss = loss + (YO(21) * RCS(12)); \
    loss = loss + (YO(21) * RCS(14)); \
    loss = loss + (YO(25) * RCS(24)); \
    loss = loss + (YO(25) * RCS(26)); \
    loss = loss + (YO(26) * RCS(34)); \
    loss = loss + (YO(27) * RCS(42)); \
    loss = loss + (YO(26) * RCS(45)); \
    loss = loss + (YO(29) * RCS(68)); \
    loss = loss + (YO(23) * RCS(78)); \
    loss = loss + (YO(31) * RCS(94)); \
    loss = loss + (YO(31) * RCS(96)); \
    loss = loss + (YO(30) * RCS(124)); \
    loss = loss + (YO(30) * RCS(126)); \
    loss = loss + (YO(30) * RCS(128)); \
    loss = loss + (YO(32) * RCS(156)); \
    loss = loss + (YO(36) * RCS(166)); \
    loss = loss + (YO(36) * RCS(170)); \
    loss = loss + (YO(39) * RCS(192)); \
    loss = loss + (YO(39) * RCS(196)); \
    loss = loss + (YO(40) * RCS(216)); \
    loss = loss + (YO(40) * RCS(218)); \
    loss = loss + SOUR(4); \
    rhs2 = -(dt * WM(3) * loss); \
    ppp = rho - FACE_SUM(3); \
    fnew = sor2 * YO(3) + (rhs1 - FACE_NBR(3)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(3) - fnew); \
    UC_UPDATE_TAIL(3); \
    prod = (YN(2) * (YN(1) * RCT(1, 6))); \
    prod = prod + (YN(3) * (YN(0) * RCT(1, 7))); \
    prod = prod + (YN(2) * (YO(5) * RCT(1, 8))); \
    prod = prod + (YN(3) * (YO(5) * RCT(1, 9))); \
    prod = prod + (YN(3) * (YO(5) * RCT(1, 9))); \
    prod = prod + (YO(5) * RCT(1, 10)); \
    prod = prod + (YN(3) * (YN(2) * RCT(1, 11))); \
    TM_WAIT(0); \
    TM_LD(1, 0, 132); \
    TM_LD(1, 1, 138); \
    TM_LD(1, 2, 154); \
    TM_LD(1, 3, 156); \
    TM_LD(1, 4, 178); \
    TM_LD(1, 5, 188); \
    TM_LD(1, 6, 192); \
    TM_LD(1, 7, 218); \
    TM_LD(1, 8, 234); \
    TM_LD(1, 9, 238); \
    TM_LD(1, 10, 274); \
    TM_LD(1, 11, 276); \
    prod = prod + (YO(6) * RCT(0, 0)); \
    prod = prod + (YN(2) * (YO(6) * RCT(0, 1))); \
    prod = prod + (YN(2) * (YO(6) * RCT(0, 1))); \
    prod = prod + (YN(3) * (YO(6) * RCT(0, 2))); \
    prod = prod + (YN(1) * (YO(5) * RCT(0, 3))); \
    prod = prod + (YO(7) * RCT(0, 4)); \
    prod = prod + (YO(7) * RCT(0, 4)); \
    prod = prod + (YN(2) * (YO(7) * RCT(0, 5))); \
    prod = prod + ((YO(5) * YO(6)) * RCT(0, 6)); \
    prod = prod + (YN(3) * (YO(7) * RCT(0, 7))); \
    prod = prod + (YN(2) * (YO(9) * RCT(0, 8))); \
    prod = prod + ((YO(8) * YO(6)) * RCT(0, 9)); \
    prod = prod + (YN(3) * (YO(10) * RCT(0, 10))); \
    prod = prod + ((YO(8) * YO(5)) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 292); \
    TM_LD(0, 1, 298); \
    TM_LD(0, 2, 316); \
    TM_LD(0, 3, 338); \
    TM_LD(0, 4, 356); \
    TM_LD(0, 5, 392); \
    TM_LD(0, 6, 422); \
    TM_LD(0, 7, 2); \
    TM_LD(0, 8, 6); \
    TM_LD(0, 9, 8); \
    TM_LD(0, 10, 14); \
    TM_LD(0, 11, 20); \
    prod = prod + (YN(3) * (YO(11) * RCT(1, 0))); \
    prod = prod + ((YO(10) * YO(5)) * RCT(1, 1)); \
    prod = prod + ((YO(5) * YO(13)) * RCT(1, 2)); \
    prod = prod + (YN(3) * (YO(12) * RCT(1, 3))); \
    prod = prod + ((YO(15) * YO(5)) * RCT(1, 4)); \
    prod = prod + ((YO(13) * YO(6)) * RCT(1, 5)); \
    prod = prod + (YN(1) * (YO(13) * RCT(1, 6))); \
    prod = prod + (YN(2) * (YO(11) * RCT(1, 7))); \
    prod = prod + (YN(1) * (YO(15) * RCS(0))); \
    prod = prod + (YN(2) * (YO(11) * RCT(1, 8))); \
    prod = prod + ((YO(20) * YO(5)) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(14) * RCS(4))); \
    prod = prod + ((YO(11) * YO(5)) * RCT(1, 10)); \
    prod = prod + (YN(3) * (YO(17) * RCT(1, 11))); \
    TM_WAIT(0); \
    TM_LD(1, 0, 30); \
    TM_LD(1, 1, 32); \
    TM_LD(1, 2, 42); \
    TM_LD(1, 3, 54); \
    TM_LD(1, 4, 56); \
    TM_LD(1, 5, 60); \
    TM_LD(1, 6, 74); \
    TM_LD(1, 7, 76); \
    TM_LD(1, 8, 82); \
    TM_LD(1, 9, 84); \
    TM_LD(1, 10, 90); \
    TM_LD(1, 11, 106); \
    prod = prod + (YN(3) * (YO(19) * RCT(0, 0))); \
    prod = prod + ((YO(18) * YO(5)) * RCT(0, 1)); \
    prod = prod + (YN(3) * (YO(18) * RCT(0, 2))); \
    prod = prod + ((YO(22) * YO(5)) * RCT(0, 3)); \
    prod = prod + ((YO(16) * YO(6)) * RCT(0, 4)); \
    prod = prod + (YN(2) * (YO(25) * RCS(19))); \
    prod = prod + ((YO(27) * YO(5)) * RCS(21)); \
    prod = prod + (YN(3) * (YO(25) * RCS(26))); \
    prod = prod + (YN(2) * ((YO(10) * YO(8)) * RCS(33))); \
    prod = prod + (YN(1) * (YO(26) * RCS(36))); \
    prod = prod + (YN(2) * (YO(26) * RCS(41))); \
    prod = prod + (YN(2) * (YO(28) * RCS(52))); \
    prod = prod + ((YO(11) * YO(5)) * RCS(55)); \
    prod = prod + ((YO(28) * YO(8)) * RCS(59)); \
    prod = prod + ((YO(28) * YO(5)) * RCS(61)); \
    prod = prod + ((YO(17) * YO(5)) * RCS(63)); \
    prod = prod + (YN(3) * (YO(29) * RCS(68))); \
    prod = prod + (YO(29) * RCT(0, 5)); \
    prod = prod + ((YO(25) * YO(5)) * RCS(81)); \
    prod = prod + (YN(1) * (YO(23) * RCS(82))); \
    prod = prod + ((YO(23) * YO(6)) * RCS(86)); \
    prod = prod + ((YO(34) * YO(5)) * RCS(91)); \
    prod = prod + ((YO(23) * YO(5)) * RCS(93)); \
    prod = prod + (YN(3) * (YO(31) * RCS(94))); \
    prod = prod + (YN(3) * (YO(31) * RCS(96))); \
    prod = prod + ((YO(33) * YO(5)) * RCS(113)); \
    prod = prod + ((YO(32) * YO(5)) * RCS(115)); \
    prod = prod + ((YO(35) * YO(5)) * RCS(117)); \
    prod = prod + (YN(3) * (YO(30) * RCS(124))); \
    prod = prod + (YN(3) * (YO(30) * RCS(126))); \
    prod = prod + (YN(3) * (YO(30) * RCS(128))); \
    prod = prod + (YO(33) * RCT(0, 6)); \
    prod = prod + ((YO(18) * YO(6)) * RCS(142)); \
    prod = prod + ((YO(31) * YO(5)) * RCS(153)); \
    prod = prod + (YN(3) * (YO(32) * RCS(156))); \
    prod = prod + ((YO(32) * YO(6)) * RCS(162)); \
    prod = prod + ((YO(32) * YO(6)) * RCS(162)); \
    prod = prod + ((YO(31) * YO(5)) * RCS(165)); \
    prod = prod + ((YO(37) * YO(5)) * RCS(175)); \
    prod = prod + ((YO(36) * YO(5)) * RCS(185)); \
    prod = prod + ((YO(37) * YO(6)) * RCS(188)); \
    prod = prod + ((YO(38) * YO(5)) * RCS(195)); \
    prod = prod + ((YO(38) * YO(6)) * RCS(202)); \
    prod = prod + (YN(3) * (YO(40) * RCS(216))); \
    prod = prod + (YN(3) * (YO(40) * RCS(218))); \
    prod = prod + ((YO(42) * YO(5)) * RCS(221)); \
    prod = prod + ((YO(41) * YO(5)) * RCS(223)); \
    prod = prod + (YN(2) * ((YO(44) * YO(38)) * RCS(239))); \
    prod = prod + (((YO(5) * YO(48)) * YO(18)) * RCS(257)); \
    prod = prod + 0.0; \
    prod = prod + 0.0; \
    prod = prod + 0.0; \
    prod = prod + (((YO(5) * YO(39)) * YO(22)) * RCS(262)); \
    prod = prod + (YN(2) * ((YO(5) * YO(43)) * RCS(280))); \
    extra = 0.0; \
    rhs1 = rho * Y0(4) + dt * WM(4) * (prod + extra); \
    loss = (YN(3) * RCT(0, 7)); \
    loss = loss + (YN(2) * RCT(0, 8)); \
    loss = loss + (YN(0) * RCT(0, 9)); \
    loss = loss + (YO(4) * RCT(0, 10)); \
    loss = loss + (YO(4) * RCT(0, 10)); \
    loss = loss + (YN(2) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 112); \
    TM_LD(0, 1, 134); \
    TM_LD(0, 2, 136); \
    TM_LD(0, 3, 152); \
    TM_LD(0, 4, 158); \
    TM_LD(0, 5, 176); \
    TM_LD(0, 6, 190); \
    TM_LD(0, 7, 194); \
    TM_LD(0, 8, 216); \
    TM_LD(0, 9, 232); \
    TM_LD(0, 10, 236); \
    TM_LD(0, 11, 272); \
    loss = loss + RCT(1, 0); \
    loss = loss + (YN(3) * RCT(1, 1)); \
    loss = loss + (YO(4) * RCT(1, 2)); \
    loss = loss + (YO(4) * RCT(1, 2)); \
    loss = loss + (YN(1) * RCT(1, 3)); \
    loss = loss + (YO(6) * RCT(1, 4)); \
    loss = loss + (YO(4) * RCT(1, 5)); \
    loss = loss + (YO(4) * RCT(1, 5)); \
    loss = loss + (YO(5) * RCT(1, 6)); \
    loss = loss + (YO(7) * RCT(1, 7)); \
    loss = loss + (YO(6) * RCT(1, 8)); \
    loss = loss + (YO(8) * RCT(1, 9)); \
    loss = loss + (YO(9) * RCT(1, 10)); \
    loss = loss + (YO(8) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 278); \
    TM_LD(1, 1, 294); \
    TM_LD(1, 2, 296); \
    TM_LD(1, 3, 318); \
    TM_LD(1, 4, 336); \
    TM_LD(1, 5, 358); \
    TM_LD(1, 6, 394); \
    TM_LD(1, 7, 420); \
    TM_LD(1, 8, 8); \
    TM_LD(1, 9, 14); \
    TM_LD(1, 10, 20); \
    TM_LD(1, 11, 48); \
    loss = loss + (YO(10) * RCT(0, 0)); \
    loss = loss + (YO(10) * RCT(0, 1)); \
    loss = loss + (YO(11) * RCT(0, 2)); \
    loss = loss + (YO(12) * RCT(0, 3)); \
    loss = loss + (YO(13) * RCT(0, 4)); \
    loss = loss + (YO(13) * RCT(0, 5)); \
    loss = loss + (YO(17) * RCT(0, 6)); \
    loss = loss + (YO(11) * RCT(0, 7)); \
    loss = loss + (YO(15) * RCT(0, 8)); \
    loss = loss + ((YO(8) * YN(2)) * RCS(1)); \
    loss = loss + (YO(14) * RCT(0, 9)); \
    loss = loss + (YO(14) * RCT(0, 10)); \
    loss = loss + ((YO(8) * YN(2)) * RCS(5)); \
    loss = loss + (YO(17) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 56); \
    TM_LD(0, 1, 72); \
    TM_LD(0, 2, 76); \
    TM_LD(0, 3, 112); \
    TM_LD(0, 4, 136); \
    TM_LD(0, 5, 152); \
    TM_LD(0, 6, 176); \
    TM_LD(0, 7, 236); \
    TM_LD(0, 8, 258); \
    TM_LD(0, 9, 268); \
    TM_LD(0, 10, 272); \
    TM_LD(0, 11, 296); \
    loss = loss + (YO(11) * RCT(1, 0)); \
    loss = loss + (YO(18) * RCT(1, 1)); \
    loss = loss + (YO(19) * RCT(1, 2)); \
    loss = loss + (YO(16) * RCT(1, 3)); \
    loss = loss + (YO(16) * RCT(1, 4)); \
    loss = loss + (YO(24) * RCT(1, 5)); \
    loss = loss + (YO(21) * RCS(18)); \
    loss = loss + (YO(21) * RCS(20)); \
    loss = loss + (YO(26) * RCS(27)); \
    loss = loss + (YO(26) * RCS(32)); \
    loss = loss + ((YO(8) * YO(8)) * RCS(37)); \
    loss = loss + (YO(27) * RCS(40)); \
    loss = loss + (YO(13) * RCS(53)); \
    loss = loss + (YO(28) * RCS(54)); \
    loss = loss + (YO(25) * RCS(58)); \
    loss = loss + (YO(29) * RCS(60)); \
    loss = loss + (YO(29) * RCS(62)); \
    loss = loss + (YO(28) * RCS(69)); \
    loss = loss + (YO(13) * RCT(1, 6)); \
    loss = loss + (YO(23) * RCS(80)); \
    loss = loss + ((YO(11) * YO(8)) * RCS(83)); \
    loss = loss + ((YO(11) * YO(10)) * RCS(87)); \
    loss = loss + (YO(31) * RCS(90)); \
    loss = loss + (YO(31) * RCS(92)); \
    loss = loss + (YO(34) * RCS(95)); \
    loss = loss + (YO(23) * RCS(97)); \
    loss = loss + (YO(30) * RCS(112)); \
    loss = loss + (YO(30) * RCS(114)); \
    loss = loss + (YO(30) * RCS(116)); \
    loss = loss + (YO(33) * RCS(125)); \
    loss = loss + (YO(32) * RCS(127)); \
    loss = loss + (YO(35) * RCS(129)); \
    loss = loss + (YO(16) * RCT(1, 7)); \
    loss = loss + (YO(35) * RCS(143)); \
    loss = loss + (YO(35) * RCS(152)); \
    loss = loss + (YO(31) * RCS(157)); \
    loss = loss + ((YO(31) * YO(4)) * RCS(163)); \
    loss = loss + ((YO(31) * YO(4)) * RCS(163)); \
    loss = loss + (YO(32) * RCS(164)); \
    loss = loss + (YO(36) * RCS(174)); \
    loss = loss + (YO(38) * RCS(184)); \
    loss = loss + ((YO(8) * YO(22)) * RCS(189)); \
    loss = loss + (YO(39) * RCS(194)); \
    loss = loss + ((YO(22) * YO(11)) * RCS(203)); \
    loss = loss + (YO(41) * RCS(217)); \
    loss = loss + (YO(42) * RCS(219)); \
    loss = loss + (YO(40) * RCS(220)); \
    loss = loss + (YO(40) * RCS(222)); \
    loss = loss + (YO(43) * RCS(238)); \
    loss = loss + (YO(46) * RCS(256)); \
    loss = loss + (YO(46) * RCS(258)); \
    loss = loss + (YO(46) * RCS(259)); \
    loss = loss + (YO(46) * RCS(260)); \
    loss = loss + (YO(48) * RCS(261)); \
    loss = loss + (YO(47) * RCS(279)); \
    loss = loss + SOUR(3); \
    rhs2 = -(dt * WM(4) * loss); \
    ppp = rho - FACE_SUM(4); \
    fnew = sor2 * YO(4) + (rhs1 - FACE_NBR(4)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(4) - fnew); \
    UC_UPDATE_TAIL(4); \
    prod = (YN(4) * (YN(0) * RCT(1, 8))); \
    prod = prod + (YN(4) * (YOS(1) * RCT(1, 9))); \
    prod = prod + (YN(4) * (YN(2) * RCT(1, 10))); \
    prod = prod + (YN(2) * (YO(6) * RCT(1, 11))); \
    TM_WAIT(0); \
    TM_LD(1, 0, 336); \
    TM_LD(1, 1, 416); \
    TM_LD(1, 2, 10); \
    TM_LD(1, 3, 12); \
    TM_LD(1, 4, 22); \
    TM_LD(1, 5, 50); \
    TM_LD(1, 6, 58); \
    TM_LD(1, 7, 74); \
    TM_LD(1, 8, 78); \
    TM_LD(1, 9, 114); \
    TM_LD(1, 10, 138); \
    TM_LD(1, 11, 154); \
    prod = prod + (YN(4) * (YO(6) * RCT(0, 0))); \
    prod = prod + (YN(2) * (YO(7) * RCT(0, 1))); \
    prod = prod + (YN(4) * (YO(7) * RCT(0, 2))); \
    prod = prod + (YN(4) * (YO(10) * RCT(0, 3))); \
    prod = prod + (YN(4) * (YO(11) * RCT(0, 4))); \
    prod = prod + (YN(4) * (YO(12) * RCT(0, 5))); \
    prod = prod + (YN(4) * (YO(13) * RCT(0, 6))); \
    prod = prod + (YN(4) * (YO(14) * RCT(0, 7))); \
    prod = prod + (YN(2) * (YO(11) * RCT(0, 8))); \
    prod = prod + (YN(2) * (YO(17) * RCT(0, 9))); \
    prod = prod + (YN(4) * (YO(17) * RCT(0, 10))); \
    prod = prod + (YN(4) * (YO(19) * RCT(0, 11))); \
    TM_WAIT(1); \
    TM_LD(0, 0, 178); \
    TM_LD(0, 1, 238); \
    TM_LD(0, 2, 256); \
    TM_LD(0, 3, 270); \
    TM_LD(0, 4, 274); \
    TM_LD(0, 5, 298); \
    TM_LD(0, 6, 338); \
    TM_LD(0, 7, 418); \
    TM_LD(0, 8, 32); \
    TM_LD(0, 9, 36); \
    TM_LD(0, 10, 42); \
    TM_LD(0, 11, 46); \
    prod = prod + (YN(4) * (YO(16) * RCT(1, 0))); \
    prod = prod + (YN(4) * (YO(21) * RCS(20))); \
    prod = prod + (YN(4) * (YO(28) * RCS(54))); \
    prod = prod + (YN(4) * (YO(29) * RCS(60))); \
    prod = prod + (YN(4) * (YO(29) * RCS(62))); \
    prod = prod + (YN(4) * (YO(23) * RCS(80))); \
    prod = prod + (YN(4) * (YO(31) * RCS(90))); \
    prod = prod + (YN(4) * (YO(31) * RCS(92))); \
    prod = prod + (YO(30) * RCT(1, 1)); \
    prod = prod + (YN(4) * (YO(30) * RCS(112))); \
    prod = prod + (YN(4) * (YO(30) * RCS(114))); \
    prod = prod + (YN(4) * (YO(30) * RCS(116))); \
    prod = prod + (YN(2) * (YO(35) * RCS(150))); \
    prod = prod + (YN(4) * (YO(35) * RCS(152))); \
    prod = prod + (YN(2) * (YO(32) * RCS(158))); \
    prod = prod + (YN(4) * (YO(32) * RCS(164))); \
    prod = prod + (YN(4) * (YO(36) * RCS(174))); \
    prod = prod + (YN(4) * (YO(38) * RCS(184))); \
    prod = prod + (YN(4) * (YO(39) * RCS(194))); \
    prod = prod + (YN(4) * (YO(40) * RCS(220))); \
    prod = prod + (YN(4) * (YO(40) * RCS(222))); \
    prod = prod + (YN(4) * (YO(46) * RCS(256))); \
    prod = prod + (YN(4) * (YO(48) * RCS(261))); \
    prod = prod + (YN(4) * (YO(47) * RCS(279))); \
    extra = (1.0 * (YN(4) * (YO(46) * RCS(258)))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(259)))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    rhs1 = rho * Y0(5) + dt * WM(5) * (prod + extra); \
    loss = (YN(2) * RCT(1, 2)); \
    loss = loss + (YN(3) * RCT(1, 3)); \
    loss = loss + RCT(1, 4); \
    loss = loss + (YN(3) * RCT(1, 5)); \
    loss = loss + (YN(1) * RCT(1, 6)); \
    loss = loss + (YN(4) * RCT(1, 7)); \
    loss = loss + (YO(6) * RCT(1, 8)); \
    loss = loss + (YO(8) * RCT(1, 9)); \
    loss = loss + (YO(10) * RCT(1, 10)); \
    loss = loss + (YO(13) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 50); \
    TM_LD(1, 1, 54); \
    TM_LD(1, 2, 58); \
    TM_LD(1, 3, 66); \
    TM_LD(1, 4, 68); \
    TM_LD(1, 5, 76); \
    TM_LD(1, 6, 80); \
    TM_LD(1, 7, 90); \
    TM_LD(1, 8, 116); \
    TM_LD(1, 9, 140); \
    TM_LD(1, 10, 146); \
    TM_LD(1, 11, 160); \
    loss = loss + (YO(15) * RCT(0, 0)); \
    loss = loss + (YO(20) * RCT(0, 1)); \
    loss = loss + (YO(20) * RCT(0, 2)); \
    loss = loss + (YO(15) * RCT(0, 3)); \
    loss = loss + (YO(11) * RCT(0, 4)); \
    loss = loss + (YO(18) * RCT(0, 5)); \
    loss = loss + (YO(22) * RCT(0, 6)); \
    loss = loss + (YO(27) * RCS(21)); \
    loss = loss + (YO(11) * RCS(55)); \
    loss = loss + (YO(28) * RCS(61)); \
    loss = loss + (YO(17) * RCS(63)); \
    loss = loss + (YO(25) * RCS(81)); \
    loss = loss + (YO(34) * RCS(91)); \
    loss = loss + (YO(23) * RCS(93)); \
    loss = loss + (YO(16) * RCT(0, 7)); \
    loss = loss + (YO(33) * RCS(113)); \
    loss = loss + (YO(32) * RCS(115)); \
    loss = loss + (YO(35) * RCS(117)); \
    loss = loss + (YO(16) * RCS(151)); \
    loss = loss + (YO(31) * RCS(153)); \
    loss = loss + (YO(16) * RCS(159)); \
    loss = loss + (YO(31) * RCS(165)); \
    loss = loss + (YO(37) * RCS(175)); \
    loss = loss + (YO(36) * RCS(185)); \
    loss = loss + (YO(38) * RCS(195)); \
    loss = loss + (YO(42) * RCS(221)); \
    loss = loss + (YO(41) * RCS(223)); \
    loss = loss + ((YO(48) * YO(18)) * RCS(257)); \
    loss = loss + ((YO(39) * YO(22)) * RCS(262)); \
    loss = loss + ((YO(43) * YN(2)) * RCS(280)); \
    rhs2 = -(dt * WM(5) * loss); \
    ppp = rho - FACE_SUM(5); \
    fnew = sor2 * YO(5) + (rhs1 - FACE_NBR(5)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(5) - fnew); \
    UC_UPDATE_TAIL(5); \
    prod = (YN(4) * (YN(3) * RCT(0, 8))); \
    prod = prod + (YN(2) * (YN(1) * RCT(0, 9))); \
    prod = prod + (YN(4) * (YOS(1) * RCT(0, 10))); \
    prod = prod + (YN(1) * (YN(0) * RCT(0, 11))); \
    TM_WAIT(1); \
    TM_LD(0, 0, 166); \
    TM_LD(0, 1, 190); \
    TM_LD(0, 2, 280); \
    TM_LD(0, 3, 310); \
    TM_LD(0, 4, 324); \
    TM_LD(0, 5, 352); \
    TM_LD(0, 6, 358); \
    TM_LD(0, 7, 34); \
    TM_LD(0, 8, 38); \
    TM_LD(0, 9, 40); \
    TM_LD(0, 10, 44); \
    TM_LD(0, 11, 48); \
    prod = prod + (YN(5) * (YN(3) * RCT(1, 0))); \
    prod = prod + (YN(4) * (YN(1) * RCT(1, 1))); \
    prod = prod + (YN(5) * (YN(1) * RCT(1, 2))); \
    prod = prod + (YN(1) * (YO(7) * RCT(1, 3))); \
    prod = prod + (YN(1) * (YO(7) * RCT(1, 3))); \
    prod = prod + (YN(2) * (YO(7) * RCT(1, 4))); \
    prod = prod + (YN(4) * (YO(7) * RCT(1, 5))); \
    prod = prod + (YN(3) * (YO(7) * RCT(1, 6))); \
    prod = prod + (YN(4) * (YO(9) * RCT(1, 7))); \
    prod = prod + (YN(1) * (YO(10) * RCT(1, 8))); \
    prod = prod + (YN(1) * (YO(11) * RCT(1, 9))); \
    prod = prod + ((YO(10) * YO(7)) * RCT(1, 10)); \
    prod = prod + (YN(1) * (YO(12) * RCT(1, 11))); \
    TM_WAIT(0); \
    TM_LD(1, 0, 52); \
    TM_LD(1, 1, 56); \
    TM_LD(1, 2, 64); \
    TM_LD(1, 3, 70); \
    TM_LD(1, 4, 78); \
    TM_LD(1, 5, 82); \
    TM_LD(1, 6, 88); \
    TM_LD(1, 7, 118); \
    TM_LD(1, 8, 142); \
    TM_LD(1, 9, 144); \
    TM_LD(1, 10, 162); \
    TM_LD(1, 11, 164); \
    prod = prod + ((YO(13) * YO(7)) * RCT(0, 0)); \
    prod = prod + (YN(4) * (YO(17) * RCT(0, 1))); \
    prod = prod + (YN(1) * (YO(17) * RCT(0, 2))); \
    prod = prod + ((YO(18) * YO(7)) * RCT(0, 3)); \
    prod = prod + (YN(1) * (YO(18) * RCT(0, 4))); \
    prod = prod + (YN(1) * (YO(16) * RCT(0, 5))); \
    prod = prod + (YN(4) * (YO(24) * RCT(0, 6))); \
    prod = prod + (((YO(13) * YO(8)) * YO(7)) * RCS(9)); \
    prod = prod + (YN(1) * (YO(22) * RCS(10))); \
    prod = prod + (YN(1) * (YO(28) * RCS(56))); \
    prod = prod + ((YO(28) * YO(7)) * RCS(71)); \
    prod = prod + (YN(1) * (YO(29) * RCS(72))); \
    prod = prod + (YN(4) * ((YO(11) * YO(10)) * RCS(87))); \
    prod = prod + (YN(1) * (YO(31) * RCS(89))); \
    prod = prod + ((YO(34) * YO(7)) * RCS(107)); \
    prod = prod + ((YO(23) * YO(7)) * RCS(109)); \
    prod = prod + (YN(1) * (YO(31) * RCS(110))); \
    prod = prod + ((YO(32) * YO(7)) * RCS(137)); \
    prod = prod + ((YO(33) * YO(7)) * RCS(139)); \
    prod = prod + ((YO(35) * YO(7)) * RCS(141)); \
    prod = prod + (YN(4) * (YO(35) * RCS(143))); \
    prod = prod + (YN(1) * (YO(35) * RCS(144))); \
    prod = prod + (YN(1) * (YO(32) * RCS(154))); \
    prod = prod + (YN(4) * ((YO(31) * YOS(1)) * RCS(163))); \
    prod = prod + (YN(1) * (YO(36) * RCS(173))); \
    prod = prod + (YN(1) * (YO(38) * RCS(180))); \
    prod = prod + (YN(4) * ((YO(8) * YO(22)) * RCS(189))); \
    prod = prod + (YN(1) * (YO(39) * RCS(201))); \
    prod = prod + (YN(4) * ((YO(22) * YO(11)) * RCS(203))); \
    prod = prod + (YN(1) * (YO(40) * RCS(208))); \
    prod = prod + (YN(1) * (YO(40) * RCS(210))); \
    prod = prod + ((YO(41) * YO(7)) * RCS(225)); \
    prod = prod + ((YO(42) * YO(7)) * RCS(227)); \
    prod = prod + (YN(1) * (YO(41) * RCS(228))); \
    prod = prod + (YN(1) * (YO(42) * RCS(230))); \
    prod = prod + (YN(1) * (YO(45) * RCS(242))); \
    prod = prod + (YN(1) * (YO(45) * RCS(244))); \
    prod = prod + (((YO(21) * YO(38)) * YO(7)) * RCS(247)); \
    prod = prod + (((YO(22) * YO(36)) * YO(7)) * RCS(249)); \
    extra = 0.0; \
    rhs1 = rho * Y0(6) + dt * WM(6) * (prod + extra); \
    loss = RCT(0, 7); \
    loss = loss + RCT(0, 8); \
    loss = loss + (YN(2) * RCT(0, 9)); \
    loss = loss + (YN(2) * RCT(0, 10)); \
    loss = loss + (YN(2) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 188); \
    TM_LD(0, 1, 282); \
    TM_LD(0, 2, 308); \
    TM_LD(0, 3, 326); \
    TM_LD(0, 4, 354); \
    TM_LD(0, 5, 356); \
    TM_LD(0, 6, 60); \
    TM_LD(0, 7, 64); \
    TM_LD(0, 8, 70); \
    TM_LD(0, 9, 74); \
    TM_LD(0, 10, 78); \
    TM_LD(0, 11, 82); \
    loss = loss + (YN(3) * RCT(1, 0)); \
    loss = loss + (YN(4) * RCT(1, 1)); \
    loss = loss + (YO(6) * RCT(1, 2)); \
    loss = loss + (YO(6) * RCT(1, 2)); \
    loss = loss + (YN(0) * RCT(1, 3)); \
    loss = loss + (YN(5) * RCT(1, 4)); \
    loss = loss + (YN(4) * RCT(1, 5)); \
    loss = loss + (YO(8) * RCT(1, 6)); \
    loss = loss + (YO(8) * RCT(1, 7)); \
    loss = loss + (YO(10) * RCT(1, 8)); \
    loss = loss + (YO(11) * RCT(1, 9)); \
    loss = loss + (YO(13) * RCT(1, 10)); \
    loss = loss + (YO(12) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 144); \
    TM_LD(1, 1, 164); \
    TM_LD(1, 2, 308); \
    TM_LD(1, 3, 62); \
    TM_LD(1, 4, 66); \
    TM_LD(1, 5, 68); \
    TM_LD(1, 6, 72); \
    TM_LD(1, 7, 76); \
    TM_LD(1, 8, 80); \
    TM_LD(1, 9, 146); \
    TM_LD(1, 10, 166); \
    TM_LD(1, 11, 310); \
    loss = loss + (YO(13) * RCT(0, 0)); \
    loss = loss + (YO(11) * RCT(0, 1)); \
    loss = loss + (YO(19) * RCT(0, 2)); \
    loss = loss + (YO(16) * RCT(0, 3)); \
    loss = loss + (YO(22) * RCT(0, 4)); \
    loss = loss + (YO(16) * RCT(0, 5)); \
    loss = loss + (YO(24) * RCS(8)); \
    loss = loss + (YO(21) * RCS(11)); \
    loss = loss + (YO(11) * RCS(57)); \
    loss = loss + (YO(29) * RCS(70)); \
    loss = loss + (YO(28) * RCS(73)); \
    loss = loss + (YO(23) * RCS(86)); \
    loss = loss + (YO(23) * RCS(88)); \
    loss = loss + (YO(31) * RCS(106)); \
    loss = loss + (YO(31) * RCS(108)); \
    loss = loss + (YO(34) * RCS(111)); \
    loss = loss + (YO(30) * RCS(136)); \
    loss = loss + (YO(30) * RCS(138)); \
    loss = loss + (YO(30) * RCS(140)); \
    loss = loss + (YO(18) * RCS(142)); \
    loss = loss + (YO(31) * RCS(145)); \
    loss = loss + (YO(31) * RCS(155)); \
    loss = loss + (YO(32) * RCS(162)); \
    loss = loss + (YO(37) * RCS(172)); \
    loss = loss + (YO(36) * RCS(181)); \
    loss = loss + (YO(37) * RCS(188)); \
    loss = loss + (YO(38) * RCS(200)); \
    loss = loss + (YO(38) * RCS(202)); \
    loss = loss + (YO(41) * RCS(209)); \
    loss = loss + (YO(42) * RCS(211)); \
    loss = loss + (YO(40) * RCS(224)); \
    loss = loss + (YO(40) * RCS(226)); \
    loss = loss + (YO(39) * RCS(229)); \
    loss = loss + (YO(39) * RCS(231)); \
    loss = loss + ((YO(21) * YO(38)) * RCS(243)); \
    loss = loss + ((YO(22) * YO(36)) * RCS(245)); \
    loss = loss + (YO(45) * RCS(246)); \
    loss = loss + (YO(45) * RCS(248)); \
    rhs2 = -(dt * WM(6) * loss); \
    ppp = rho - FACE_SUM(6); \
    fnew = sor2 * YO(6) + (rhs1 - FACE_NBR(6)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(6) - fnew); \
    UC_UPDATE_TAIL(6); \
    prod = (YN(4) * (YOS(1) * RCT(0, 6))); \
    prod = prod + (YN(6) * (YOS(2) * RCT(0, 7))); \
    prod = prod + (YN(6) * (YN(0) * RCT(0, 8))); \
    prod = prod + (YN(5) * (YN(4) * RCT(0, 9))); \
    prod = prod + (YN(6) * (YN(5) * RCT(0, 10))); \
    prod = prod + (YN(6) * (YN(4) * RCT(0, 11))); \
    TM_WAIT(1); \
    TM_LD(0, 0, 86); \
    TM_LD(0, 1, 90); \
    TM_LD(0, 2, 94); \
    TM_LD(0, 3, 96); \
    TM_LD(0, 4, 100); \
    TM_LD(0, 5, 104); \
    TM_LD(0, 6, 112); \
    TM_LD(0, 7, 116); \
    TM_LD(0, 8, 120); \
    TM_LD(0, 9, 220); \
    TM_LD(0, 10, 240); \
    TM_LD(0, 11, 248); \
    prod = prod + (YN(6) * (YO(11) * RCT(1, 0))); \
    prod = prod + (YN(6) * (YO(12) * RCT(1, 1))); \
    prod = prod + (YN(6) * (YO(19) * RCT(1, 2))); \
    prod = prod + (YN(6) * (YO(24) * RCS(8))); \
    prod = prod + (YN(6) * (YO(29) * RCS(70))); \
    prod = prod + (YN(6) * (YO(31) * RCS(106))); \
    prod = prod + (YN(6) * (YO(31) * RCS(108))); \
    prod = prod + (YN(6) * (YO(30) * RCS(136))); \
    prod = prod + (YN(6) * (YO(30) * RCS(138))); \
    prod = prod + (YN(6) * (YO(30) * RCS(140))); \
    prod = prod + (YN(6) * (YO(40) * RCS(224))); \
    prod = prod + (YN(6) * (YO(40) * RCS(226))); \
    prod = prod + (YN(6) * (YO(45) * RCS(246))); \
    prod = prod + (YN(6) * (YO(45) * RCS(248))); \
    extra = 0.0; \
    rhs1 = rho * Y0(7) + dt * WM(7) * (prod + extra); \
    loss = RCT(1, 3); \
    loss = loss + (YN(1) * RCT(1, 4)); \
    loss = loss + (YN(2) * RCT(1, 5)); \
    loss = loss + (YN(2) * RCT(1, 6)); \
    loss = loss + (YN(4) * RCT(1, 7)); \
    loss = loss + (YN(3) * RCT(1, 8)); \
    loss = loss + (YO(10) * RCT(1, 9)); \
    loss = loss + (YO(13) * RCT(1, 10)); \
    loss = loss + (YO(18) * RCT(1, 11)); \
    loss = loss + ((YO(13) * YO(8)) * RCS(9)); \
    loss = loss + (YO(28) * RCS(71)); \
    loss = loss + (YO(34) * RCS(107)); \
    loss = loss + (YO(23) * RCS(109)); \
    loss = loss + (YO(32) * RCS(137)); \
    loss = loss + (YO(33) * RCS(139)); \
    loss = loss + (YO(35) * RCS(141)); \
    loss = loss + (YO(41) * RCS(225)); \
    loss = loss + (YO(42) * RCS(227)); \
    loss = loss + ((YO(21) * YO(38)) * RCS(247)); \
    loss = loss + ((YO(22) * YO(36)) * RCS(249)); \
    rhs2 = -(dt * WM(7) * loss); \
    ppp = rho - FACE_SUM(7); \
    fnew = sor2 * YO(7) + (rhs1 - FACE_NBR(7)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(7) - fnew); \
    UC_UPDATE_TAIL(7); \
    TM_WAIT(0); \
    TM_LD(1, 0, 260); \
    TM_LD(1, 1, 400); \
    TM_LD(1, 2, 408); \
    TM_LD(1, 3, 84); \
    TM_LD(1, 4, 88); \
    TM_LD(1, 5, 92); \
    TM_LD(1, 6, 98); \
    TM_LD(1, 7, 102); \
    TM_LD(1, 8, 106); \
    TM_LD(1, 9, 114); \
    TM_LD(1, 10, 118); \
    TM_LD(1, 11, 122); \
    prod = (YN(2) * (YO(9) * RCT(0, 0))); \
    prod = prod + (YN(4) * (YO(9) * RCT(0, 1))); \
    prod = prod + (YN(3) * (YO(9) * RCT(0, 2))); \
    prod = prod + (YO(10) * RCT(0, 3)); \
    prod = prod + (YN(2) * (YO(10) * RCT(0, 4))); \
    prod = prod + (YN(3) * (YO(10) * RCT(0, 5))); \
    prod = prod + (YN(4) * (YO(10) * RCT(0, 6))); \
    prod = prod + (YN(1) * (YO(10) * RCT(0, 7))); \
    prod = prod + ((YO(10) * YO(13)) * RCT(0, 8)); \
    prod = prod + (YN(1) * (YO(15) * RCS(0))); \
    prod = prod + ((YO(15) * YO(9)) * RCT(0, 9)); \
    prod = prod + (YN(3) * (YO(14) * RCS(2))); \
    prod = prod + (YN(3) * (YO(14) * RCT(0, 10))); \
    prod = prod + (YN(1) * (YO(14) * RCS(4))); \
    prod = prod + (YN(3) * (YO(20) * RCT(0, 11))); \
    TM_WAIT(1); \
    TM_LD(0, 0, 222); \
    TM_LD(0, 1, 242); \
    TM_LD(0, 2, 250); \
    TM_LD(0, 3, 262); \
    TM_LD(0, 4, 402); \
    TM_LD(0, 5, 410); \
    TM_LD(0, 6, 84); \
    TM_LD(0, 7, 88); \
    TM_LD(0, 8, 92); \
    TM_LD(0, 9, 108); \
    TM_LD(0, 10, 244); \
    TM_LD(0, 11, 86); \
    prod = prod + ((YO(20) * YO(9)) * RCT(1, 0)); \
    prod = prod + (YN(6) * (YO(24) * RCS(8))); \
    prod = prod + (YN(3) * (YO(21) * RCS(14))); \
    prod = prod + (YN(1) * (YO(21) * RCS(16))); \
    prod = prod + (YN(2) * (YO(25) * RCS(22))); \
    prod = prod + ((YO(25) * YO(13)) * RCS(28)); \
    prod = prod + (YN(2) * (YO(26) * RCS(30))); \
    prod = prod + (YN(4) * (YO(26) * RCS(32))); \
    prod = prod + (YN(3) * (YO(26) * RCS(34))); \
    prod = prod + (YN(3) * (YO(26) * RCS(34))); \
    prod = prod + (YN(1) * (YO(26) * RCS(36))); \
    prod = prod + (YN(1) * (YO(26) * RCS(36))); \
    prod = prod + (YN(1) * (YO(26) * RCS(38))); \
    prod = prod + (YN(3) * (YO(27) * RCS(42))); \
    prod = prod + (YN(1) * (YO(27) * RCS(48))); \
    prod = prod + (YN(4) * (YO(25) * RCS(58))); \
    prod = prod + (YN(1) * (YO(23) * RCS(82))); \
    prod = prod + ((YO(23) * YO(13)) * RCS(84)); \
    prod = prod + (YO(23) * RCT(1, 1)); \
    prod = prod + (YO(34) * RCT(1, 2)); \
    prod = prod + ((YO(18) * YO(9)) * RCS(147)); \
    prod = prod + (YN(3) * (YO(36) * RCS(166))); \
    prod = prod + ((YO(37) * YO(10)) * RCS(186)); \
    prod = prod + (YN(6) * (YO(37) * RCS(188))); \
    prod = prod + (YN(1) * (YO(36) * RCS(190))); \
    prod = prod + ((0.5 * SOUR(2)) * YN(1)); \
    prod = prod + (SOUR(3) * YN(4)); \
    prod = prod + (SOUR(4) * YN(3)); \
    extra = 0.0; \
    rhs1 = rho * Y0(8) + dt * WM(8) * (prod + extra); \
    loss = (YN(4) * RCT(1, 3)); \
    loss = loss + (YN(6) * RCT(1, 4)); \
    loss = loss + (YN(1) * RCT(1, 5)); \
    loss = loss + (YN(2) * RCT(1, 6)); \
    loss = loss + (YN(0) * RCT(1, 7)); \
    loss = loss + (YN(4) * RCT(1, 8)); \
    loss = loss + (YN(5) * RCT(1, 9)); \
    loss = loss + (YN(6) * RCT(1, 10)); \
    loss = loss + (YO(12) * RCT(1, 11)); \
    loss = loss + ((YN(4) * YN(2)) * RCS(1)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 90); \
    TM_LD(1, 1, 94); \
    TM_LD(1, 2, 110); \
    TM_LD(1, 3, 220); \
    TM_LD(1, 4, 246); \
    TM_LD(1, 5, 260); \
    TM_LD(1, 6, 98); \
    TM_LD(1, 7, 102); \
    TM_LD(1, 8, 106); \
    TM_LD(1, 9, 114); \
    TM_LD(1, 10, 118); \
    TM_LD(1, 11, 122); \
    loss = loss + (YO(11) * RCT(0, 0)); \
    loss = loss + ((YN(2) * YN(2)) * RCS(3)); \
    loss = loss + (YN(0) * RCT(0, 1)); \
    loss = loss + ((YN(4) * YN(2)) * RCS(5)); \
    loss = loss + (YN(2) * RCT(0, 2)); \
    loss = loss + (YO(10) * RCT(0, 3)); \
    loss = loss + ((YO(13) * YN(7)) * RCS(9)); \
    loss = loss + (YO(14) * RCS(15)); \
    loss = loss + (YO(11) * RCS(17)); \
    loss = loss + (YO(13) * RCS(23)); \
    loss = loss + (YO(18) * RCS(29)); \
    loss = loss + (YO(15) * RCS(31)); \
    loss = loss + ((YO(10) * YN(2)) * RCS(33)); \
    loss = loss + ((YO(8) * YN(2)) * RCS(35)); \
    loss = loss + ((YO(8) * YN(2)) * RCS(35)); \
    loss = loss + ((YO(8) * YN(4)) * RCS(37)); \
    loss = loss + ((YO(8) * YN(4)) * RCS(37)); \
    loss = loss + ((YO(9) * YN(2)) * RCS(39)); \
    loss = loss + (YO(20) * RCS(43)); \
    loss = loss + (YO(10) * RCS(49)); \
    loss = loss + (YO(28) * RCS(59)); \
    loss = loss + ((YO(11) * YN(4)) * RCS(83)); \
    loss = loss + ((YO(18) * YN(2)) * RCS(85)); \
    loss = loss + (YO(13) * RCT(0, 4)); \
    loss = loss + (YO(13) * RCT(0, 5)); \
    loss = loss + (YO(35) * RCS(146)); \
    loss = loss + (YO(16) * RCS(167)); \
    loss = loss + (YO(36) * RCS(187)); \
    loss = loss + ((YN(4) * YO(22)) * RCS(189)); \
    loss = loss + ((YO(13) * YO(10)) * RCS(191)); \
    rhs2 = -(dt * WM(8) * loss); \
    ppp = rho - FACE_SUM(8); \
    fnew = sor2 * YO(8) + (rhs1 - FACE_NBR(8)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(8) - fnew); \
    UC_UPDATE_TAIL(8); \
    prod = (YN(8) * (YN(4) * RCT(0, 6))); \
    prod = prod + (YN(8) * (YN(6) * RCT(0, 7))); \
    prod = prod + (YN(8) * (YN(1) * RCT(0, 8))); \
    prod = prod + (YN(3) * (YO(10) * RCT(0, 9))); \
    prod = prod + (YN(8) * (YO(11) * RCT(0, 0))); \
    prod = prod + (YN(1) * (YO(14) * RCT(0, 10))); \
    prod = prod + (YN(8) * (YO(10) * RCT(0, 3))); \
    prod = prod + (YN(3) * (YO(25) * RCS(24))); \
    prod = prod + (YN(1) * (YO(26) * RCS(38))); \
    prod = prod + (YN(1) * (YO(27) * RCS(46))); \
    prod = prod + (YN(8) * (YO(35) * RCS(146))); \
    extra = 0.0; \
    rhs1 = rho * Y0(9) + dt * WM(9) * (prod + extra); \
    loss = (YN(2) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 126); \
    TM_LD(0, 1, 128); \
    TM_LD(0, 2, 132); \
    TM_LD(0, 3, 136); \
    TM_LD(0, 4, 140); \
    TM_LD(0, 5, 144); \
    TM_LD(0, 6, 252); \
    TM_LD(0, 7, 260); \
    TM_LD(0, 8, 340); \
    TM_LD(0, 9, 376); \
    TM_LD(0, 10, 404); \
    TM_LD(0, 11, 96); \
    loss = loss + (YN(4) * RCT(1, 0)); \
    loss = loss + (YN(3) * RCT(1, 1)); \
    loss = loss + (YN(2) * RCT(1, 2)); \
    loss = loss + (YO(15) * RCT(1, 3)); \
    loss = loss + (YN(0) * RCT(1, 4)); \
    loss = loss + (YO(20) * RCT(1, 5)); \
    loss = loss + (YO(14) * RCS(25)); \
    loss = loss + ((YN(8) * YN(2)) * RCS(39)); \
    loss = loss + (YO(20) * RCS(47)); \
    loss = loss + (YO(18) * RCS(147)); \
    rhs2 = -(dt * WM(9) * loss); \
    ppp = rho - FACE_SUM(9); \
    fnew = sor2 * YO(9) + (rhs1 - FACE_NBR(9)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(9) - fnew); \
    UC_UPDATE_TAIL(9); \
    prod = (YN(8) * (YN(2) * RCT(1, 6))); \
    prod = prod + (YN(8) * (YN(0) * RCT(1, 7))); \
    prod = prod + (YN(8) * (YN(4) * RCT(1, 8))); \
    prod = prod + (YN(9) * (YN(2) * RCT(1, 2))); \
    prod = prod + (YN(8) * (YN(5) * RCT(1, 9))); \
    prod = prod + (YN(8) * (YN(6) * RCT(1, 10))); \
    prod = prod + (YN(8) * (YO(12) * RCT(1, 11))); \
    TM_WAIT(0); \
    TM_LD(1, 0, 100); \
    TM_LD(1, 1, 104); \
    TM_LD(1, 2, 108); \
    TM_LD(1, 3, 112); \
    TM_LD(1, 4, 116); \
    TM_LD(1, 5, 120); \
    TM_LD(1, 6, 124); \
    TM_LD(1, 7, 130); \
    TM_LD(1, 8, 134); \
    TM_LD(1, 9, 138); \
    TM_LD(1, 10, 142); \
    TM_LD(1, 11, 146); \
    prod = prod + (YO(11) * RCT(0, 0)); \
    prod = prod + (YN(2) * (YO(11) * RCT(0, 1))); \
    prod = prod + (YN(3) * (YO(11) * RCT(0, 2))); \
    prod = prod + (YN(4) * (YO(11) * RCT(0, 3))); \
    prod = prod + (YN(1) * (YO(11) * RCT(0, 4))); \
    prod = prod + (YN(6) * (YO(11) * RCT(0, 5))); \
    prod = prod + (YN(1) * (YO(20) * RCT(0, 6))); \
    prod = prod + (YN(9) * (YO(20) * RCT(0, 7))); \
    prod = prod + (YN(3) * (YO(16) * RCT(0, 8))); \
    prod = prod + (YN(1) * (YO(22) * RCT(0, 9))); \
    prod = prod + (YN(4) * (YO(26) * RCS(32))); \
    prod = prod + (YN(1) * (YO(27) * RCS(48))); \
    prod = prod + (YN(2) * (YO(23) * RCS(74))); \
    prod = prod + (YN(3) * (YO(23) * RCS(78))); \
    prod = prod + (YN(6) * (YO(23) * RCS(86))); \
    prod = prod + (YO(31) * RCT(0, 10)); \
    prod = prod + (YN(1) * (YO(37) * RCS(176))); \
    prod = prod + (YN(8) * (YO(36) * RCS(187))); \
    prod = prod + (YN(1) * (YO(36) * RCS(190))); \
    prod = prod + (YN(3) * (YO(39) * RCS(192))); \
    extra = 0.0; \
    rhs1 = rho * Y0(10) + dt * WM(10) * (prod + extra); \
    loss = RCT(0, 11); \
    TM_WAIT(1); \
    TM_LD(0, 0, 254); \
    TM_LD(0, 1, 262); \
    TM_LD(0, 2, 342); \
    TM_LD(0, 3, 378); \
    TM_LD(0, 4, 406); \
    TM_LD(0, 5, 124); \
    TM_LD(0, 6, 130); \
    TM_LD(0, 7, 134); \
    TM_LD(0, 8, 138); \
    TM_LD(0, 9, 142); \
    TM_LD(0, 10, 146); \
    TM_LD(0, 11, 180); \
    loss = loss + (YN(2) * RCT(1, 0)); \
    loss = loss + (YN(3) * RCT(1, 1)); \
    loss = loss + (YN(3) * RCT(1, 2)); \
    loss = loss + (YN(4) * RCT(1, 3)); \
    loss = loss + (YN(1) * RCT(1, 4)); \
    loss = loss + (YO(13) * RCT(1, 5)); \
    loss = loss + (YN(2) * RCT(1, 6)); \
    loss = loss + (YN(0) * RCT(1, 7)); \
    loss = loss + (YN(4) * RCT(1, 8)); \
    loss = loss + (YN(5) * RCT(1, 9)); \
    loss = loss + (YN(6) * RCT(1, 10)); \
    loss = loss + (YN(7) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 192); \
    TM_LD(1, 1, 216); \
    TM_LD(1, 2, 220); \
    TM_LD(1, 3, 232); \
    TM_LD(1, 4, 256); \
    TM_LD(1, 5, 264); \
    TM_LD(1, 6, 272); \
    TM_LD(1, 7, 276); \
    TM_LD(1, 8, 280); \
    TM_LD(1, 9, 284); \
    TM_LD(1, 10, 320); \
    TM_LD(1, 11, 376); \
    loss = loss + (YN(3) * RCT(0, 0)); \
    loss = loss + (YN(8) * RCT(0, 1)); \
    loss = loss + (YO(13) * RCT(0, 2)); \
    loss = loss + (YO(11) * RCT(0, 3)); \
    loss = loss + ((YN(8) * YN(2)) * RCS(33)); \
    loss = loss + (YN(8) * RCS(49)); \
    loss = loss + (YO(13) * RCS(75)); \
    loss = loss + (YO(11) * RCS(79)); \
    loss = loss + ((YO(11) * YN(4)) * RCS(87)); \
    loss = loss + (YO(13) * RCT(0, 4)); \
    loss = loss + (YO(25) * RCS(177)); \
    loss = loss + (YO(37) * RCS(186)); \
    loss = loss + ((YO(13) * YN(8)) * RCS(191)); \
    loss = loss + (YO(18) * RCS(193)); \
    rhs2 = -(dt * WM(10) * loss); \
    ppp = rho - FACE_SUM(10); \
    fnew = sor2 * YO(10) + (rhs1 - FACE_NBR(10)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(10) - fnew); \
    UC_UPDATE_TAIL(10); \
    prod = (YN(10) * (YN(2) * RCT(0, 5))); \
    prod = prod + (YN(10) * (YN(0) * RCT(0, 6))); \
    prod = prod + (YN(10) * (YN(4) * RCT(0, 7))); \
    prod = prod + (YN(10) * (YN(5) * RCT(0, 8))); \
    prod = prod + (YN(10) * (YN(6) * RCT(0, 9))); \
    prod = prod + (YN(10) * (YN(7) * RCT(0, 10))); \
    prod = prod + (YN(3) * (YO(13) * RCT(0, 11))); \
    TM_WAIT(1); \
    TM_LD(0, 0, 384); \
    TM_LD(0, 1, 428); \
    TM_LD(0, 2, 126); \
    TM_LD(0, 3, 128); \
    TM_LD(0, 4, 132); \
    TM_LD(0, 5, 136); \
    TM_LD(0, 6, 140); \
    TM_LD(0, 7, 144); \
    TM_LD(0, 8, 182); \
    TM_LD(0, 9, 194); \
    TM_LD(0, 10, 218); \
    TM_LD(0, 11, 222); \
    prod = prod + (YN(1) * (YO(13) * RCT(1, 0))); \
    prod = prod + (YN(4) * (YO(15) * RCT(1, 1))); \
    prod = prod + (YN(9) * (YO(15) * RCT(1, 2))); \
    prod = prod + (YN(4) * (YO(14) * RCT(1, 3))); \
    prod = prod + (YN(5) * (YO(20) * RCT(1, 4))); \
    prod = prod + (YN(2) * (YO(17) * RCT(1, 5))); \
    prod = prod + (YN(4) * (YO(17) * RCT(1, 6))); \
    prod = prod + (YN(3) * (YO(17) * RCT(1, 7))); \
    prod = prod + (YN(1) * (YO(17) * RCT(1, 8))); \
    prod = prod + (YO(17) * RCT(1, 9)); \
    prod = prod + (YN(3) * (YO(18) * RCT(1, 10))); \
    prod = prod + (YN(1) * (YO(22) * RCT(1, 11))); \
    prod = prod + (YN(1) * (YO(21) * RCS(16))); \
    prod = prod + (YN(2) * (YO(28) * RCS(50))); \
    prod = prod + (YN(4) * (YO(28) * RCS(54))); \
    prod = prod + (YN(1) * (YO(28) * RCS(56))); \
    TM_WAIT(0); \
    TM_LD(1, 0, 234); \
    TM_LD(1, 1, 258); \
    TM_LD(1, 2, 266); \
    TM_LD(1, 3, 274); \
    TM_LD(1, 4, 278); \
    TM_LD(1, 5, 282); \
    TM_LD(1, 6, 286); \
    TM_LD(1, 7, 322); \
    TM_LD(1, 8, 378); \
    TM_LD(1, 9, 386); \
    TM_LD(1, 10, 430); \
    TM_LD(1, 11, 120); \
    prod = prod + (YO(28) * RCT(0, 0)); \
    prod = prod + (YN(3) * (YO(23) * RCS(78))); \
    prod = prod + (YN(1) * (YO(23) * RCS(82))); \
    prod = prod + (YN(6) * (YO(23) * RCS(86))); \
    prod = prod + (YO(35) * RCT(0, 1)); \
    prod = prod + (YN(6) * (YO(38) * RCS(202))); \
    extra = 0.0; \
    rhs1 = rho * Y0(11) + dt * WM(11) * (prod + extra); \
    loss = RCT(0, 2); \
    loss = loss + (YN(2) * RCT(0, 3)); \
    loss = loss + (YN(3) * RCT(0, 4)); \
    loss = loss + (YN(4) * RCT(0, 5)); \
    loss = loss + (YN(1) * RCT(0, 6)); \
    loss = loss + (YN(6) * RCT(0, 7)); \
    loss = loss + (YN(2) * RCT(0, 8)); \
    loss = loss + (YN(4) * RCT(0, 9)); \
    loss = loss + (YN(2) * RCT(0, 10)); \
    loss = loss + (YN(8) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 150); \
    TM_LD(0, 1, 154); \
    TM_LD(0, 2, 158); \
    TM_LD(0, 3, 162); \
    TM_LD(0, 4, 166); \
    TM_LD(0, 5, 208); \
    TM_LD(0, 6, 300); \
    TM_LD(0, 7, 122); \
    TM_LD(0, 8, 148); \
    TM_LD(0, 9, 152); \
    TM_LD(0, 10, 156); \
    TM_LD(0, 11, 160); \
    loss = loss + (YN(2) * RCT(1, 0)); \
    loss = loss + (YN(2) * RCT(1, 1)); \
    loss = loss + (YN(0) * RCT(1, 2)); \
    loss = loss + (YN(5) * RCT(1, 3)); \
    loss = loss + (YN(4) * RCT(1, 4)); \
    loss = loss + (YN(6) * RCT(1, 5)); \
    loss = loss + (YN(2) * RCT(1, 6)); \
    loss = loss + (YO(13) * RCT(1, 7)); \
    loss = loss + (YN(10) * RCT(1, 8)); \
    loss = loss + (YN(8) * RCS(17)); \
    loss = loss + (YN(0) * RCS(51)); \
    loss = loss + (YN(5) * RCS(55)); \
    loss = loss + (YN(6) * RCS(57)); \
    loss = loss + (YN(2) * RCT(1, 9)); \
    loss = loss + (YN(10) * RCS(79)); \
    loss = loss + ((YN(8) * YN(4)) * RCS(83)); \
    loss = loss + ((YN(10) * YN(4)) * RCS(87)); \
    loss = loss + (YO(13) * RCT(1, 10)); \
    loss = loss + ((YN(4) * YO(22)) * RCS(203)); \
    rhs2 = -(dt * WM(11) * loss); \
    ppp = rho - FACE_SUM(11); \
    fnew = sor2 * YO(11) + (rhs1 - FACE_NBR(11)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(11) - fnew); \
    UC_UPDATE_TAIL(11); \
    prod = (YN(10) * (YO(13) * RCT(1, 11))); \
    TM_WAIT(0); \
    TM_LD(1, 0, 164); \
    TM_LD(1, 1, 210); \
    TM_LD(1, 2, 302); \
    TM_LD(1, 3, 122); \
    TM_LD(1, 4, 148); \
    TM_LD(1, 5, 152); \
    TM_LD(1, 6, 156); \
    TM_LD(1, 7, 160); \
    TM_LD(1, 8, 170); \
    TM_LD(1, 9, 174); \
    TM_LD(1, 10, 178); \
    TM_LD(1, 11, 182); \
    prod = prod + (YN(0) * (YO(13) * RCT(0, 0))); \
    prod = prod + (YN(5) * (YO(13) * RCT(0, 1))); \
    prod = prod + (YN(4) * (YO(13) * RCT(0, 2))); \
    prod = prod + (YN(6) * (YO(13) * RCT(0, 3))); \
    prod = prod + (YN(7) * (YO(13) * RCT(0, 4))); \
    prod = prod + (YN(2) * (YO(13) * RCT(0, 5))); \
    prod = prod + ((YO(19) * YO(13)) * RCT(0, 6)); \
    prod = prod + ((YO(31) * YO(13)) * RCS(102)); \
    prod = prod + ((YO(31) * YO(13)) * RCS(104)); \
    prod = prod + ((YO(30) * YO(13)) * RCS(130)); \
    prod = prod + ((YO(30) * YO(13)) * RCS(132)); \
    prod = prod + ((YO(30) * YO(13)) * RCS(134)); \
    prod = prod + ((YO(38) * YO(13)) * RCS(182)); \
    prod = prod + ((YO(43) * YO(13)) * RCS(240)); \
    extra = 0.0; \
    rhs1 = rho * Y0(12) + dt * WM(12) * (prod + extra); \
    loss = (YN(8) * RCT(0, 7)); \
    loss = loss + (YN(2) * RCT(0, 8)); \
    loss = loss + (YN(4) * RCT(0, 9)); \
    loss = loss + (YN(3) * RCT(0, 10)); \
    loss = loss + (YN(1) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 186); \
    TM_LD(0, 1, 190); \
    TM_LD(0, 2, 194); \
    TM_LD(0, 3, 198); \
    TM_LD(0, 4, 202); \
    TM_LD(0, 5, 206); \
    TM_LD(0, 6, 210); \
    TM_LD(0, 7, 214); \
    TM_LD(0, 8, 302); \
    TM_LD(0, 9, 320); \
    TM_LD(0, 10, 340); \
    TM_LD(0, 11, 392); \
    loss = loss + (YN(6) * RCT(1, 0)); \
    loss = loss + RCT(1, 1); \
    loss = loss + (YO(18) * RCT(1, 2)); \
    loss = loss + (YO(34) * RCS(103)); \
    loss = loss + (YO(23) * RCS(105)); \
    loss = loss + (YO(33) * RCS(131)); \
    loss = loss + (YO(32) * RCS(133)); \
    loss = loss + (YO(35) * RCS(135)); \
    loss = loss + (YO(36) * RCS(183)); \
    loss = loss + ((YO(21) * YO(22)) * RCS(241)); \
    rhs2 = -(dt * WM(12) * loss); \
    ppp = rho - FACE_SUM(12); \
    fnew = sor2 * YO(12) + (rhs1 - FACE_NBR(12)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(12) - fnew); \
    UC_UPDATE_TAIL(12); \
    prod = (YN(12) * (YN(8) * RCT(1, 3))); \
    prod = prod + (YN(12) * (YN(2) * RCT(1, 4))); \
    prod = prod + (YN(12) * (YN(4) * RCT(1, 5))); \
    prod = prod + (YN(12) * (YN(3) * RCT(1, 6))); \
    prod = prod + (YN(12) * (YN(1) * RCT(1, 7))); \
    prod = prod + (YN(12) * (YN(6) * RCT(1, 0))); \
    prod = prod + (YN(0) * (YO(14) * RCT(1, 8))); \
    prod = prod + (YN(0) * (YO(15) * RCT(1, 9))); \
    prod = prod + (YN(5) * (YO(15) * RCT(1, 10))); \
    prod = prod + (YN(11) * (YN(2) * RCT(1, 11))); \
    TM_WAIT(0); \
    TM_LD(1, 0, 400); \
    TM_LD(1, 1, 404); \
    TM_LD(1, 2, 408); \
    TM_LD(1, 3, 412); \
    TM_LD(1, 4, 428); \
    TM_LD(1, 5, 446); \
    TM_LD(1, 6, 454); \
    TM_LD(1, 7, 456); \
    TM_LD(1, 8, 468); \
    TM_LD(1, 9, 486); \
    TM_LD(1, 10, 508); \
    TM_LD(1, 11, 120); \
    prod = prod + (YN(2) * (YO(16) * RCT(0, 0))); \
    prod = prod + (YN(4) * (YO(17) * RCT(0, 1))); \
    prod = prod + (YN(11) * (YN(4) * RCT(0, 2))); \
    prod = prod + (YN(3) * (YO(17) * RCT(0, 3))); \
    prod = prod + (YN(0) * (YO(16) * RCT(0, 4))); \
    prod = prod + (YN(0) * (YO(16) * RCT(0, 4))); \
    prod = prod + (YN(2) * (YO(18) * RCT(0, 5))); \
    prod = prod + (YN(2) * (YO(18) * RCT(0, 5))); \
    prod = prod + (YN(12) * RCT(0, 6)); \
    prod = prod + (YO(19) * RCT(0, 7)); \
    prod = prod + (YO(19) * RCT(0, 7)); \
    prod = prod + (YN(12) * (YO(18) * RCT(0, 8))); \
    prod = prod + (YN(3) * (YO(18) * RCT(0, 9))); \
    prod = prod + (YN(3) * (YO(16) * RCT(0, 10))); \
    prod = prod + (YN(6) * (YO(24) * RCS(8))); \
    prod = prod + (YN(2) * (YO(25) * RCS(22))); \
    prod = prod + (YN(8) * (YO(18) * RCS(29))); \
    prod = prod + (YN(2) * (YO(28) * RCS(52))); \
    prod = prod + (YO(29) * RCT(0, 11)); \
    prod = prod + (YN(2) * (YO(23) * RCS(74))); \
    prod = prod + (YN(8) * ((YO(18) * YN(2)) * RCS(85))); \
    TM_WAIT(1); \
    TM_LD(0, 0, 150); \
    TM_LD(0, 1, 154); \
    TM_LD(0, 2, 158); \
    TM_LD(0, 3, 162); \
    TM_LD(0, 4, 166); \
    TM_LD(0, 5, 168); \
    TM_LD(0, 6, 172); \
    TM_LD(0, 7, 176); \
    TM_LD(0, 8, 180); \
    TM_LD(0, 9, 184); \
    TM_LD(0, 10, 188); \
    TM_LD(0, 11, 192); \
    prod = prod + (YO(23) * RCT(1, 0)); \
    prod = prod + (YO(31) * RCT(1, 1)); \
    prod = prod + (YO(34) * RCT(1, 2)); \
    prod = prod + (YN(12) * (YO(34) * RCS(103))); \
    prod = prod + (YN(12) * (YO(23) * RCS(105))); \
    prod = prod + (YO(30) * RCT(1, 3)); \
    prod = prod + (YN(12) * (YO(33) * RCS(131))); \
    prod = prod + (YN(12) * (YO(32) * RCS(133))); \
    prod = prod + (YN(12) * (YO(35) * RCS(135))); \
    prod = prod + (YO(35) * RCT(1, 4)); \
    prod = prod + (YN(2) * (YO(35) * RCS(148))); \
    prod = prod + (YN(2) * (YO(32) * RCS(160))); \
    prod = prod + (YN(2) * (YO(36) * RCS(169))); \
    prod = prod + (YN(3) * (YO(36) * RCS(170))); \
    prod = prod + (YN(12) * (YO(36) * RCS(183))); \
    prod = prod + (YO(38) * RCT(1, 5)); \
    prod = prod + (YN(1) * (YO(36) * RCS(190))); \
    prod = prod + (YN(3) * (YO(39) * RCS(196))); \
    prod = prod + (YO(39) * RCT(1, 6)); \
    prod = prod + (YN(2) * (YO(39) * RCS(204))); \
    prod = prod + (YN(2) * (YO(38) * RCS(207))); \
    prod = prod + (YO(40) * RCT(1, 7)); \
    prod = prod + (YO(42) * RCT(1, 8)); \
    prod = prod + (YN(12) * ((YO(21) * YO(22)) * RCS(241))); \
    prod = prod + (YO(43) * RCT(1, 9)); \
    prod = prod + (YN(2) * (YO(48) * RCS(265))); \
    prod = prod + (YN(2) * (YO(48) * RCS(271))); \
    prod = prod + (YO(47) * RCT(1, 10)); \
    prod = prod + (YN(2) * (YO(47) * RCS(275))); \
    extra = (1.0 * (YO(46) * RCS(250))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(252)))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(253)))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(258)))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    rhs1 = rho * Y0(13) + dt * WM(13) * (prod + extra); \
    loss = (YN(10) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 196); \
    TM_LD(1, 1, 200); \
    TM_LD(1, 2, 204); \
    TM_LD(1, 3, 208); \
    TM_LD(1, 4, 212); \
    TM_LD(1, 5, 300); \
    TM_LD(1, 6, 322); \
    TM_LD(1, 7, 342); \
    TM_LD(1, 8, 394); \
    TM_LD(1, 9, 402); \
    TM_LD(1, 10, 406); \
    TM_LD(1, 11, 410); \
    loss = loss + (YN(0) * RCT(0, 0)); \
    loss = loss + (YN(5) * RCT(0, 1)); \
    loss = loss + (YN(4) * RCT(0, 2)); \
    loss = loss + (YN(6) * RCT(0, 3)); \
    loss = loss + (YN(7) * RCT(0, 4)); \
    loss = loss + (YN(2) * RCT(0, 5)); \
    loss = loss + (YN(2) * RCT(0, 6)); \
    loss = loss + (YN(4) * RCT(0, 7)); \
    loss = loss + (YN(3) * RCT(0, 8)); \
    loss = loss + (YO(14) * RCT(0, 9)); \
    loss = loss + (YN(6) * RCT(0, 10)); \
    loss = loss + (YN(1) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 414); \
    TM_LD(0, 1, 430); \
    TM_LD(0, 2, 444); \
    TM_LD(0, 3, 452); \
    TM_LD(0, 4, 458); \
    TM_LD(0, 5, 470); \
    TM_LD(0, 6, 484); \
    TM_LD(0, 7, 510); \
    TM_LD(0, 8, 168); \
    TM_LD(0, 9, 186); \
    TM_LD(0, 10, 224); \
    TM_LD(0, 11, 230); \
    loss = loss + (YN(1) * RCT(1, 0)); \
    loss = loss + (YO(13) * RCT(1, 1)); \
    loss = loss + (YO(13) * RCT(1, 1)); \
    loss = loss + (YO(13) * RCT(1, 2)); \
    loss = loss + (YO(13) * RCT(1, 2)); \
    loss = loss + (YN(2) * RCT(1, 3)); \
    loss = loss + (YO(13) * RCT(1, 4)); \
    loss = loss + (YO(13) * RCT(1, 4)); \
    loss = loss + (YO(19) * RCT(1, 5)); \
    loss = loss + (YN(11) * RCT(1, 6)); \
    loss = loss + (YN(10) * RCT(1, 7)); \
    loss = loss + ((YN(8) * YN(7)) * RCS(9)); \
    loss = loss + (YN(8) * RCS(23)); \
    loss = loss + (YO(25) * RCS(28)); \
    loss = loss + (YN(4) * RCS(53)); \
    loss = loss + (YN(4) * RCT(1, 8)); \
    loss = loss + (YN(10) * RCS(75)); \
    loss = loss + (YO(23) * RCS(84)); \
    loss = loss + (YN(8) * RCT(1, 9)); \
    loss = loss + (YN(10) * RCT(1, 10)); \
    loss = loss + (YN(8) * RCT(1, 11)); \
    loss = loss + (YO(31) * RCS(102)); \
    loss = loss + (YO(31) * RCS(104)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 234); \
    TM_LD(1, 1, 238); \
    TM_LD(1, 2, 242); \
    TM_LD(1, 3, 246); \
    TM_LD(1, 4, 170); \
    TM_LD(1, 5, 184); \
    TM_LD(1, 6, 226); \
    TM_LD(1, 7, 228); \
    TM_LD(1, 8, 232); \
    TM_LD(1, 9, 236); \
    TM_LD(1, 10, 240); \
    TM_LD(1, 11, 244); \
    loss = loss + (YO(28) * RCT(0, 0)); \
    loss = loss + (YO(30) * RCS(130)); \
    loss = loss + (YO(30) * RCS(132)); \
    loss = loss + (YO(30) * RCS(134)); \
    loss = loss + (YN(11) * RCT(0, 1)); \
    loss = loss + (YO(28) * RCS(149)); \
    loss = loss + (YO(28) * RCS(161)); \
    loss = loss + (YO(21) * RCS(168)); \
    loss = loss + (YO(26) * RCS(171)); \
    loss = loss + (YO(38) * RCS(182)); \
    loss = loss + (YO(21) * RCT(0, 2)); \
    loss = loss + ((YN(10) * YN(8)) * RCS(191)); \
    loss = loss + ((YO(25) * YN(2)) * RCS(197)); \
    loss = loss + (YO(22) * RCT(0, 3)); \
    loss = loss + (YO(16) * RCS(205)); \
    loss = loss + (YO(22) * RCS(206)); \
    loss = loss + (YO(18) * RCT(0, 4)); \
    loss = loss + (YO(16) * RCT(0, 5)); \
    loss = loss + (YO(43) * RCS(240)); \
    loss = loss + (YO(37) * RCT(0, 6)); \
    loss = loss + ((YO(16) * YO(16)) * RCS(266)); \
    loss = loss + ((YN(0) * YO(43)) * RCS(272)); \
    loss = loss + (YO(38) * RCT(0, 7)); \
    loss = loss + (YO(39) * RCS(276)); \
    rhs2 = -(dt * WM(13) * loss); \
    ppp = rho - FACE_SUM(13); \
    fnew = sor2 * YO(13) + (rhs1 - FACE_NBR(13)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(13) - fnew); \
    UC_UPDATE_TAIL(13); \
    prod = (YN(13) * (YN(2) * RCT(0, 8))); \
    prod = prod + (YN(2) * (YO(16) * RCT(0, 9))); \
    prod = prod + (YO(15) * RCT(0, 10)); \
    prod = prod + (YN(0) * (YO(20) * RCT(0, 11))); \
    TM_WAIT(1); \
    TM_LD(0, 0, 172); \
    TM_LD(0, 1, 176); \
    TM_LD(0, 2, 218); \
    TM_LD(0, 3, 222); \
    TM_LD(0, 4, 226); \
    TM_LD(0, 5, 268); \
    TM_LD(0, 6, 174); \
    TM_LD(0, 7, 178); \
    TM_LD(0, 8, 216); \
    TM_LD(0, 9, 220); \
    TM_LD(0, 10, 224); \
    TM_LD(0, 11, 270); \
    prod = prod + (YN(11) * (YN(2) * RCT(1, 0))); \
    prod = prod + (YN(5) * (YO(20) * RCT(1, 1))); \
    prod = prod + (YN(8) * ((YN(2) * YN(2)) * RCS(3))); \
    prod = prod + (YN(8) * (YN(0) * RCT(1, 2))); \
    prod = prod + (YN(9) * (YN(0) * RCT(1, 3))); \
    prod = prod + (YN(8) * ((YN(4) * YN(2)) * RCS(5))); \
    prod = prod + (YN(2) * ((YO(21) * YOS(0)) * RCS(7))); \
    prod = prod + (YN(2) * ((YO(21) * YOS(0)) * RCS(7))); \
    prod = prod + (YN(3) * (YO(21) * RCS(14))); \
    prod = prod + (YN(3) * (YO(25) * RCS(24))); \
    extra = 0.0; \
    rhs1 = rho * Y0(14) + dt * WM(14) * (prod + extra); \
    loss = (YN(0) * RCT(1, 4)); \
    loss = loss + (YN(13) * RCT(1, 5)); \
    loss = loss + RCT(1, 6); \
    loss = loss + (YN(2) * RCT(1, 7)); \
    loss = loss + (YN(4) * RCT(1, 8)); \
    loss = loss + (YN(4) * RCT(1, 9)); \
    loss = loss + (YN(3) * RCS(2)); \
    loss = loss + (YN(3) * RCT(1, 10)); \
    loss = loss + (YN(1) * RCT(1, 11)); \
    loss = loss + (YN(1) * RCS(4)); \
    loss = loss + (YO(14) * RCS(6)); \
    loss = loss + (YO(14) * RCS(6)); \
    loss = loss + (YN(8) * RCS(15)); \
    loss = loss + (YN(9) * RCS(25)); \
    rhs2 = -(dt * WM(14) * loss); \
    ppp = rho - FACE_SUM(14); \
    fnew = sor2 * YO(14) + (rhs1 - FACE_NBR(14)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(14) - fnew); \
    UC_UPDATE_TAIL(14); \
    TM_WAIT(0); \
    TM_LD(1, 0, 184); \
    TM_LD(1, 1, 200); \
    TM_LD(1, 2, 312); \
    TM_LD(1, 3, 316); \
    TM_LD(1, 4, 324); \
    TM_LD(1, 5, 328); \
    TM_LD(1, 6, 334); \
    TM_LD(1, 7, 338); \
    TM_LD(1, 8, 342); \
    TM_LD(1, 9, 346); \
    TM_LD(1, 10, 350); \
    TM_LD(1, 11, 354); \
    prod = (YN(13) * (YN(2) * RCT(0, 0))); \
    prod = prod + (YN(13) * (YN(4) * RCT(0, 1))); \
    prod = prod + (YN(11) * (YN(2) * RCT(0, 2))); \
    prod = prod + (YN(8) * ((YN(4) * YN(2)) * RCS(1))); \
    prod = prod + (YN(11) * (YN(8) * RCT(0, 3))); \
    prod = prod + (YN(14) * RCT(0, 4)); \
    prod = prod + (YN(2) * (YO(17) * RCT(0, 5))); \
    prod = prod + (YN(2) * (YO(26) * RCS(30))); \
    extra = 0.0; \
    rhs1 = rho * Y0(15) + dt * WM(15) * (prod + extra); \
    loss = (YN(0) * RCT(0, 6)); \
    loss = loss + (YN(5) * RCT(0, 7)); \
    loss = loss + (YN(4) * RCT(0, 8)); \
    loss = loss + (YN(1) * RCS(0)); \
    loss = loss + (YN(9) * RCT(0, 9)); \
    loss = loss + RCT(0, 10); \
    loss = loss + (YN(5) * RCT(0, 11)); \
    loss = loss + (YN(8) * RCS(31)); \
    rhs2 = -(dt * WM(15) * loss); \
    ppp = rho - FACE_SUM(15); \
    fnew = sor2 * YO(15) + (rhs1 - FACE_NBR(15)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(15) - fnew); \
    UC_UPDATE_TAIL(15); \
    TM_WAIT(1); \
    TM_LD(0, 0, 358); \
    TM_LD(0, 1, 362); \
    TM_LD(0, 2, 366); \
    TM_LD(0, 3, 416); \
    TM_LD(0, 4, 422); \
    TM_LD(0, 5, 468); \
    TM_LD(0, 6, 492); \
    TM_LD(0, 7, 504); \
    TM_LD(0, 8, 186); \
    TM_LD(0, 9, 202); \
    TM_LD(0, 10, 314); \
    TM_LD(0, 11, 318); \
    prod = (YN(14) * (YN(13) * RCT(1, 0))); \
    prod = prod + (YN(13) * (YOS(3) * RCT(1, 1))); \
    prod = prod + (YN(2) * (YO(18) * RCT(1, 2))); \
    prod = prod + (YN(3) * (YO(18) * RCT(1, 3))); \
    prod = prod + (YN(1) * (YO(18) * RCT(1, 4))); \
    prod = prod + (YO(18) * RCT(1, 5)); \
    prod = prod + (YN(0) * (YO(22) * RCT(1, 6))); \
    prod = prod + (YN(5) * (YO(22) * RCT(1, 7))); \
    prod = prod + (YN(13) * (YN(10) * RCT(1, 8))); \
    prod = prod + (YN(2) * (YO(23) * RCT(1, 9))); \
    prod = prod + ((YO(22) * YO(18)) * RCT(1, 10)); \
    prod = prod + ((YO(22) * YO(18)) * RCT(1, 10)); \
    prod = prod + (YN(6) * (YO(22) * RCT(1, 11))); \
    TM_WAIT(0); \
    TM_LD(1, 0, 326); \
    TM_LD(1, 1, 330); \
    TM_LD(1, 2, 332); \
    TM_LD(1, 3, 336); \
    TM_LD(1, 4, 340); \
    TM_LD(1, 5, 344); \
    TM_LD(1, 6, 348); \
    TM_LD(1, 7, 352); \
    TM_LD(1, 8, 356); \
    TM_LD(1, 9, 360); \
    TM_LD(1, 10, 364); \
    TM_LD(1, 11, 418); \
    prod = prod + (YN(4) * (YO(24) * RCT(0, 0))); \
    prod = prod + (YN(2) * (YO(22) * RCT(0, 1))); \
    prod = prod + (YN(0) * (YO(21) * RCT(0, 2))); \
    prod = prod + (YO(30) * RCT(0, 3)); \
    prod = prod + (YO(33) * RCT(0, 4)); \
    prod = prod + (YN(2) * (YO(35) * RCS(150))); \
    prod = prod + (YN(2) * (YO(32) * RCS(158))); \
    prod = prod + (YN(3) * (YO(36) * RCS(166))); \
    prod = prod + (YN(2) * (YO(39) * RCS(204))); \
    prod = prod + (YO(42) * RCT(0, 5)); \
    prod = prod + (YN(2) * (YO(43) * RCS(234))); \
    prod = prod + (YO(45) * RCT(0, 6)); \
    prod = prod + (YO(48) * RCT(0, 7)); \
    prod = prod + (YN(2) * (YO(48) * RCS(265))); \
    prod = prod + (YN(2) * (YO(48) * RCS(265))); \
    prod = prod + (YN(2) * (YO(48) * RCS(269))); \
    prod = prod + (YN(2) * (YO(47) * RCS(273))); \
    prod = prod + (YN(2) * (YO(47) * RCS(277))); \
    extra = (1.0 * (YO(46) * RCS(250))); \
    extra = extra + (1.0 * (YO(46) * RCS(250))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(251)))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(252)))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(253)))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(253)))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(253)))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(258)))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(259)))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    rhs1 = rho * Y0(16) + dt * WM(16) * (prod + extra); \
    loss = (YN(2) * RCT(0, 8)); \
    loss = loss + (YN(0) * RCT(0, 9)); \
    loss = loss + (YN(0) * RCT(0, 10)); \
    loss = loss + (YN(4) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 420); \
    TM_LD(0, 1, 470); \
    TM_LD(0, 2, 494); \
    TM_LD(0, 3, 506); \
    TM_LD(0, 4, 188); \
    TM_LD(0, 5, 196); \
    TM_LD(0, 6, 266); \
    TM_LD(0, 7, 270); \
    TM_LD(0, 8, 274); \
    TM_LD(0, 9, 278); \
    TM_LD(0, 10, 282); \
    TM_LD(0, 11, 286); \
    loss = loss + (YN(6) * RCT(1, 0)); \
    loss = loss + (YN(2) * RCT(1, 1)); \
    loss = loss + (YN(2) * RCT(1, 2)); \
    loss = loss + (YN(4) * RCT(1, 3)); \
    loss = loss + (YN(3) * RCT(1, 4)); \
    loss = loss + (YN(3) * RCT(1, 5)); \
    loss = loss + (YO(16) * RCT(1, 6)); \
    loss = loss + (YO(16) * RCT(1, 6)); \
    loss = loss + (YN(1) * RCT(1, 7)); \
    loss = loss + (YN(6) * RCT(1, 8)); \
    loss = loss + RCT(1, 9); \
    loss = loss + RCT(1, 10); \
    loss = loss + (YN(5) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 390); \
    TM_LD(1, 1, 190); \
    TM_LD(1, 2, 198); \
    TM_LD(1, 3, 264); \
    TM_LD(1, 4, 268); \
    TM_LD(1, 5, 272); \
    TM_LD(1, 6, 276); \
    TM_LD(1, 7, 280); \
    TM_LD(1, 8, 284); \
    TM_LD(1, 9, 388); \
    TM_LD(1, 10, 204); \
    TM_LD(1, 11, 288); \
    loss = loss + (YN(4) * RCT(0, 0)); \
    loss = loss + (YN(5) * RCS(151)); \
    loss = loss + (YN(5) * RCS(159)); \
    loss = loss + (YN(8) * RCS(167)); \
    loss = loss + (YN(13) * RCS(205)); \
    loss = loss + (YN(13) * RCT(0, 1)); \
    loss = loss + (YO(22) * RCS(235)); \
    loss = loss + (YO(36) * RCT(0, 2)); \
    loss = loss + (YO(39) * RCT(0, 3)); \
    loss = loss + ((YO(16) * YN(13)) * RCS(266)); \
    loss = loss + ((YO(16) * YN(13)) * RCS(266)); \
    loss = loss + ((YN(0) * YO(38)) * RCS(270)); \
    loss = loss + (YO(18) * RCS(274)); \
    loss = loss + ((YN(0) * YO(22)) * RCS(278)); \
    rhs2 = -(dt * WM(16) * loss); \
    ppp = rho - FACE_SUM(16); \
    fnew = sor2 * YO(16) + (rhs1 - FACE_NBR(16)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(16) - fnew); \
    UC_UPDATE_TAIL(16); \
    prod = (YN(13) * (YN(6) * RCT(0, 4))); \
    prod = prod + (YN(13) * (YN(1) * RCT(0, 5))); \
    prod = prod + (YN(11) * (YN(0) * RCT(0, 6))); \
    prod = prod + (YN(15) * (YN(5) * RCT(0, 7))); \
    prod = prod + (YN(11) * (YN(5) * RCT(0, 8))); \
    prod = prod + (YN(11) * (YN(4) * RCT(0, 9))); \
    prod = prod + (YN(11) * (YN(6) * RCT(0, 10))); \
    prod = prod + (YN(11) * (YN(2) * RCT(0, 11))); \
    TM_WAIT(1); \
    TM_LD(0, 0, 292); \
    TM_LD(0, 1, 296); \
    TM_LD(0, 2, 300); \
    TM_LD(0, 3, 304); \
    TM_LD(0, 4, 308); \
    TM_LD(0, 5, 314); \
    TM_LD(0, 6, 318); \
    TM_LD(0, 7, 322); \
    TM_LD(0, 8, 326); \
    TM_LD(0, 9, 330); \
    TM_LD(0, 10, 348); \
    TM_LD(0, 11, 456); \
    prod = prod + (YO(28) * RCT(1, 0)); \
    prod = prod + (YN(4) * (YO(29) * RCS(62))); \
    prod = prod + (YN(2) * (YO(29) * RCS(66))); \
    extra = 0.0; \
    rhs1 = rho * Y0(17) + dt * WM(17) * (prod + extra); \
    loss = (YN(4) * RCT(1, 1)); \
    loss = loss + (YN(3) * RCT(1, 2)); \
    loss = loss + (YN(2) * RCT(1, 3)); \
    loss = loss + (YN(2) * RCT(1, 4)); \
    loss = loss + (YN(4) * RCT(1, 5)); \
    loss = loss + (YN(3) * RCT(1, 6)); \
    loss = loss + (YN(1) * RCT(1, 7)); \
    loss = loss + RCT(1, 8); \
    loss = loss + RCT(1, 9); \
    loss = loss + (YN(5) * RCS(63)); \
    loss = loss + (YN(0) * RCS(67)); \
    rhs2 = -(dt * WM(17) * loss); \
    ppp = rho - FACE_SUM(17); \
    fnew = sor2 * YO(17) + (rhs1 - FACE_NBR(17)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(17) - fnew); \
    UC_UPDATE_TAIL(17); \
    prod = (YN(13) * (YOS(3) * RCT(1, 10))); \
    prod = prod + (YN(2) * (YO(19) * RCT(1, 11))); \
    TM_WAIT(0); \
    TM_LD(1, 0, 500); \
    TM_LD(1, 1, 206); \
    TM_LD(1, 2, 290); \
    TM_LD(1, 3, 294); \
    TM_LD(1, 4, 298); \
    TM_LD(1, 5, 302); \
    TM_LD(1, 6, 306); \
    TM_LD(1, 7, 310); \
    TM_LD(1, 8, 312); \
    TM_LD(1, 9, 316); \
    TM_LD(1, 10, 320); \
    TM_LD(1, 11, 324); \
    prod = prod + (YN(3) * (YO(19) * RCT(0, 0))); \
    prod = prod + (YN(4) * (YO(19) * RCT(0, 1))); \
    prod = prod + (YN(13) * (YO(19) * RCT(0, 2))); \
    prod = prod + (YO(19) * RCT(0, 3)); \
    prod = prod + (YN(6) * (YO(19) * RCT(0, 4))); \
    prod = prod + (YN(16) * (YN(0) * RCT(0, 5))); \
    prod = prod + (YN(16) * (YN(4) * RCT(0, 6))); \
    prod = prod + (YN(13) * (YN(11) * RCT(0, 7))); \
    prod = prod + (YN(16) * (YN(6) * RCT(0, 8))); \
    prod = prod + (YN(16) * (YN(2) * RCT(0, 9))); \
    prod = prod + (YN(16) * (YOS(4) * RCT(0, 10))); \
    prod = prod + (YN(13) * (YO(25) * RCS(28))); \
    prod = prod + (YN(13) * (YO(23) * RCS(84))); \
    prod = prod + (YN(4) * (YO(35) * RCS(143))); \
    prod = prod + (YN(8) * (YO(35) * RCS(146))); \
    prod = prod + (YN(3) * (YO(39) * RCS(192))); \
    prod = prod + (YO(40) * RCT(0, 11)); \
    prod = prod + (YN(2) * (YO(46) * RCS(254))); \
    prod = prod + (YN(4) * (YO(46) * RCS(256))); \
    TM_WAIT(1); \
    TM_LD(0, 0, 328); \
    TM_LD(0, 1, 350); \
    TM_LD(0, 2, 458); \
    TM_LD(0, 3, 502); \
    TM_LD(0, 4, 212); \
    TM_LD(0, 5, 290); \
    TM_LD(0, 6, 294); \
    TM_LD(0, 7, 298); \
    TM_LD(0, 8, 302); \
    TM_LD(0, 9, 306); \
    TM_LD(0, 10, 310); \
    TM_LD(0, 11, 214); \
    prod = prod + (YO(48) * RCT(1, 0)); \
    prod = prod + (YN(2) * (YO(48) * RCS(267))); \
    prod = prod + (YN(2) * (YO(47) * RCS(273))); \
    extra = (1.0 * (YO(46) * RCS(250))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(251)))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(259)))); \
    rhs1 = rho * Y0(18) + dt * WM(18) * (prod + extra); \
    loss = (YN(2) * RCT(1, 1)); \
    loss = loss + (YN(0) * RCT(1, 2)); \
    loss = loss + (YN(4) * RCT(1, 3)); \
    loss = loss + (YN(5) * RCT(1, 4)); \
    loss = loss + (YN(12) * RCT(1, 5)); \
    loss = loss + (YN(2) * RCT(1, 6)); \
    loss = loss + (YN(7) * RCT(1, 7)); \
    loss = loss + (YN(2) * RCT(1, 8)); \
    loss = loss + (YN(3) * RCT(1, 9)); \
    loss = loss + (YN(3) * RCT(1, 10)); \
    loss = loss + (YN(1) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 288); \
    TM_LD(1, 1, 292); \
    TM_LD(1, 2, 296); \
    TM_LD(1, 3, 300); \
    TM_LD(1, 4, 304); \
    TM_LD(1, 5, 308); \
    TM_LD(1, 6, 228); \
    TM_LD(1, 7, 236); \
    TM_LD(1, 8, 250); \
    TM_LD(1, 9, 254); \
    TM_LD(1, 10, 258); \
    TM_LD(1, 11, 262); \
    loss = loss + RCT(0, 0); \
    loss = loss + (YO(22) * RCT(0, 1)); \
    loss = loss + (YN(8) * RCS(29)); \
    loss = loss + ((YN(8) * YN(2)) * RCS(85)); \
    loss = loss + (YN(6) * RCS(142)); \
    loss = loss + (YN(9) * RCS(147)); \
    loss = loss + (YN(10) * RCS(193)); \
    loss = loss + (YN(13) * RCT(0, 2)); \
    loss = loss + ((YN(0) * YO(48)) * RCS(255)); \
    loss = loss + ((YN(5) * YO(48)) * RCS(257)); \
    loss = loss + (YO(38) * RCT(0, 3)); \
    loss = loss + (YO(39) * RCS(268)); \
    loss = loss + (YN(16) * RCS(274)); \
    rhs2 = -(dt * WM(18) * loss); \
    ppp = rho - FACE_SUM(18); \
    fnew = sor2 * YO(18) + (rhs1 - FACE_NBR(18)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(18) - fnew); \
    UC_UPDATE_TAIL(18); \
    prod = (YN(13) * (YOS(3) * RCT(0, 4))); \
    prod = prod + (YN(18) * (YN(0) * RCT(0, 5))); \
    prod = prod + (YN(18) * (YN(4) * RCT(0, 6))); \
    prod = prod + (YN(18) * (YN(5) * RCT(0, 7))); \
    prod = prod + (YN(18) * (YN(12) * RCT(0, 8))); \
    prod = prod + (YN(18) * (YN(2) * RCT(0, 9))); \
    prod = prod + (YN(18) * (YN(7) * RCT(0, 10))); \
    extra = 0.0; \
    rhs1 = rho * Y0(19) + dt * WM(19) * (prod + extra); \
    loss = RCT(0, 11); \
    TM_WAIT(1); \
    TM_LD(0, 0, 230); \
    TM_LD(0, 1, 238); \
    TM_LD(0, 2, 248); \
    TM_LD(0, 3, 252); \
    TM_LD(0, 4, 256); \
    TM_LD(0, 5, 260); \
    TM_LD(0, 6, 364); \
    TM_LD(0, 7, 368); \
    TM_LD(0, 8, 372); \
    TM_LD(0, 9, 446); \
    TM_LD(0, 10, 488); \
    TM_LD(0, 11, 366); \
    loss = loss + (YN(2) * RCT(1, 0)); \
    loss = loss + (YN(3) * RCT(1, 1)); \
    loss = loss + (YN(4) * RCT(1, 2)); \
    loss = loss + (YN(13) * RCT(1, 3)); \
    loss = loss + RCT(1, 4); \
    loss = loss + (YN(6) * RCT(1, 5)); \
    rhs2 = -(dt * WM(19) * loss); \
    ppp = rho - FACE_SUM(19); \
    fnew = sor2 * YO(19) + (rhs1 - FACE_NBR(19)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(19) - fnew); \
    UC_UPDATE_TAIL(19); \
    prod = (YN(14) * (YN(2) * RCT(1, 6))); \
    prod = prod + (YN(14) * (YN(4) * RCT(1, 7))); \
    prod = prod + (YN(8) * (YN(2) * RCT(1, 8))); \
    prod = prod + (YN(10) * (YN(3) * RCT(1, 9))); \
    prod = prod + (YN(11) * (YN(2) * RCT(1, 10))); \
    prod = prod + (YN(10) * (YN(8) * RCT(1, 11))); \
    prod = prod + (YN(3) * (YO(27) * RCS(42))); \
    prod = prod + (YN(1) * (YO(27) * RCS(46))); \
    extra = 0.0; \
    rhs1 = rho * Y0(20) + dt * WM(20) * (prod + extra); \
    TM_WAIT(0); \
    TM_LD(1, 0, 370); \
    TM_LD(1, 1, 374); \
    TM_LD(1, 2, 444); \
    TM_LD(1, 3, 490); \
    TM_LD(1, 4, 332); \
    TM_LD(1, 5, 336); \
    TM_LD(1, 6, 348); \
    TM_LD(1, 7, 352); \
    TM_LD(1, 8, 360); \
    TM_LD(1, 9, 378); \
    TM_LD(1, 10, 382); \
    TM_LD(1, 11, 454); \
    loss = (YN(0) * RCT(0, 0)); \
    loss = loss + (YN(5) * RCT(0, 1)); \
    loss = loss + (YN(3) * RCT(0, 2)); \
    loss = loss + (YN(1) * RCT(0, 3)); \
    loss = loss + (YN(5) * RCT(0, 4)); \
    loss = loss + (YN(9) * RCT(0, 5)); \
    loss = loss + (YN(8) * RCS(43)); \
    loss = loss + (YN(9) * RCS(47)); \
    rhs2 = -(dt * WM(20) * loss); \
    ppp = rho - FACE_SUM(20); \
    fnew = sor2 * YO(20) + (rhs1 - FACE_NBR(20)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(20) - fnew); \
    UC_UPDATE_TAIL(20); \
    prod = (YN(14) * (YOS(5) * RCS(6))); \
    prod = prod + (YN(16) * RCT(0, 6)); \
    prod = prod + (YN(2) * (YO(22) * RCT(0, 7))); \
    prod = prod + (YO(22) * RCT(0, 8)); \
    prod = prod + (YN(1) * (YO(22) * RCS(10))); \
    prod = prod + (YN(2) * (YO(26) * RCS(13))); \
    prod = prod + (YN(14) * (YN(8) * RCS(15))); \
    prod = prod + (YN(11) * (YN(8) * RCS(17))); \
    prod = prod + (YN(2) * (YO(25) * RCS(19))); \
    prod = prod + (YN(5) * (YO(27) * RCS(21))); \
    prod = prod + (YN(2) * (YO(36) * RCS(169))); \
    prod = prod + (YO(38) * RCT(0, 9)); \
    prod = prod + (YO(43) * RCS(232)); \
    prod = prod + (YN(2) * (YO(43) * RCS(236))); \
    prod = prod + (YN(13) * (YO(43) * RCS(240))); \
    prod = prod + (YO(45) * RCT(0, 10)); \
    prod = prod + (YN(1) * (YO(45) * RCS(242))); \
    prod = prod + (YN(6) * (YO(45) * RCS(246))); \
    extra = 0.0; \
    rhs1 = rho * Y0(21) + dt * WM(21) * (prod + extra); \
    loss = ((YN(2) * YN(2)) * RCS(7)); \
    loss = loss + (YN(0) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 476); \
    TM_LD(0, 1, 482); \
    TM_LD(0, 2, 496); \
    TM_LD(0, 3, 334); \
    TM_LD(0, 4, 338); \
    TM_LD(0, 5, 350); \
    TM_LD(0, 6, 354); \
    TM_LD(0, 7, 362); \
    TM_LD(0, 8, 368); \
    TM_LD(0, 9, 372); \
    TM_LD(0, 10, 376); \
    TM_LD(0, 11, 380); \
    loss = loss + (YN(0) * RCT(1, 0)); \
    loss = loss + (YN(2) * RCT(1, 1)); \
    loss = loss + (YN(6) * RCS(11)); \
    loss = loss + (YN(3) * RCS(12)); \
    loss = loss + (YN(3) * RCS(14)); \
    loss = loss + (YN(1) * RCS(16)); \
    loss = loss + (YN(4) * RCS(18)); \
    loss = loss + (YN(4) * RCS(20)); \
    loss = loss + (YN(13) * RCS(168)); \
    loss = loss + (YN(13) * RCT(1, 2)); \
    loss = loss + ((YO(22) * YN(2)) * RCS(233)); \
    loss = loss + ((YN(0) * YO(22)) * RCS(237)); \
    loss = loss + ((YN(12) * YO(22)) * RCS(241)); \
    loss = loss + (YO(39) * RCT(1, 3)); \
    loss = loss + ((YO(38) * YN(6)) * RCS(243)); \
    loss = loss + ((YO(38) * YN(7)) * RCS(247)); \
    loss = loss + SOUR(0); \
    rhs2 = -(dt * WM(21) * loss); \
    ppp = rho - FACE_SUM(21); \
    fnew = sor2 * YO(21) + (rhs1 - FACE_NBR(21)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(21) - fnew); \
    UC_UPDATE_TAIL(21); \
    prod = (YN(16) * (YN(2) * RCT(1, 4))); \
    prod = prod + (YN(16) * (YN(4) * RCT(1, 5))); \
    prod = prod + (YN(16) * (YOS(4) * RCT(1, 6))); \
    prod = prod + (YN(16) * (YN(1) * RCT(1, 7))); \
    prod = prod + (YN(16) * RCT(1, 8)); \
    prod = prod + (YN(21) * (YN(0) * RCT(1, 0))); \
    prod = prod + (YN(21) * (YN(2) * RCT(1, 1))); \
    prod = prod + (YN(11) * (YN(10) * RCT(1, 9))); \
    prod = prod + (YN(3) * (YO(23) * RCT(1, 10))); \
    prod = prod + (YN(21) * (YN(6) * RCS(11))); \
    prod = prod + (YN(6) * (YO(37) * RCS(188))); \
    prod = prod + (YN(6) * (YO(38) * RCS(202))); \
    prod = prod + (YO(39) * RCT(1, 11)); \
    prod = prod + (YN(2) * (YO(38) * RCS(207))); \
    prod = prod + (YO(43) * RCS(232)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 452); \
    TM_LD(1, 1, 478); \
    TM_LD(1, 2, 480); \
    TM_LD(1, 3, 498); \
    TM_LD(1, 4, 344); \
    TM_LD(1, 5, 380); \
    TM_LD(1, 6, 398); \
    TM_LD(1, 7, 402); \
    TM_LD(1, 8, 346); \
    TM_LD(1, 9, 382); \
    TM_LD(1, 10, 396); \
    TM_LD(1, 11, 400); \
    prod = prod + (YO(43) * RCT(0, 0)); \
    prod = prod + (YO(43) * RCT(0, 0)); \
    prod = prod + (YO(43) * RCT(0, 1)); \
    prod = prod + (YO(43) * RCT(0, 1)); \
    prod = prod + (YN(2) * (YO(43) * RCS(234))); \
    prod = prod + (YN(2) * (YO(43) * RCS(236))); \
    prod = prod + (YN(13) * (YO(43) * RCS(240))); \
    prod = prod + (YO(45) * RCT(0, 2)); \
    prod = prod + (YN(1) * (YO(45) * RCS(244))); \
    prod = prod + (YN(6) * (YO(45) * RCS(248))); \
    prod = prod + (YN(4) * (YO(48) * RCS(261))); \
    prod = prod + (YN(2) * (YO(48) * RCS(263))); \
    prod = prod + (YN(2) * (YO(47) * RCS(277))); \
    extra = 0.0; \
    rhs1 = rho * Y0(22) + dt * WM(22) * (prod + extra); \
    loss = (YN(0) * RCT(0, 3)); \
    loss = loss + (YN(5) * RCT(0, 4)); \
    loss = loss + (YN(18) * RCT(0, 5)); \
    loss = loss + (YN(6) * RCT(0, 6)); \
    loss = loss + (YN(2) * RCT(0, 7)); \
    loss = loss + (YN(2) * RCT(0, 8)); \
    loss = loss + RCT(0, 9); \
    loss = loss + (YN(1) * RCT(0, 10)); \
    loss = loss + (YN(1) * RCT(0, 11)); \
    loss = loss + (YN(1) * RCS(10)); \
    loss = loss + ((YN(4) * YN(8)) * RCS(189)); \
    loss = loss + ((YN(4) * YN(11)) * RCS(203)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 356); \
    TM_LD(0, 1, 358); \
    TM_LD(0, 2, 396); \
    TM_LD(0, 3, 398); \
    TM_LD(0, 4, 386); \
    TM_LD(0, 5, 388); \
    TM_LD(0, 6, 412); \
    TM_LD(0, 7, 384); \
    TM_LD(0, 8, 390); \
    TM_LD(0, 9, 414); \
    TM_LD(0, 10, 394); \
    TM_LD(0, 11, 392); \
    loss = loss + (YN(13) * RCT(1, 0)); \
    loss = loss + (YN(13) * RCS(206)); \
    loss = loss + ((YN(21) * YN(2)) * RCS(233)); \
    loss = loss + (YO(22) * RCT(1, 1)); \
    loss = loss + (YO(22) * RCT(1, 1)); \
    loss = loss + (YO(22) * RCT(1, 2)); \
    loss = loss + (YO(22) * RCT(1, 2)); \
    loss = loss + (YN(16) * RCS(235)); \
    loss = loss + ((YN(0) * YN(21)) * RCS(237)); \
    loss = loss + ((YN(12) * YN(21)) * RCS(241)); \
    loss = loss + (YO(38) * RCT(1, 3)); \
    loss = loss + ((YO(36) * YN(6)) * RCS(245)); \
    loss = loss + ((YO(36) * YN(7)) * RCS(249)); \
    loss = loss + ((YN(5) * YO(39)) * RCS(262)); \
    loss = loss + ((YN(0) * YO(39)) * RCS(264)); \
    loss = loss + ((YN(0) * YN(16)) * RCS(278)); \
    rhs2 = -(dt * WM(22) * loss); \
    ppp = rho - FACE_SUM(22); \
    fnew = sor2 * YO(22) + (rhs1 - FACE_NBR(22)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(22) - fnew); \
    UC_UPDATE_TAIL(22); \
    prod = (YN(16) * (YN(3) * RCT(1, 4))); \
    prod = prod + (YN(22) * (YN(1) * RCT(1, 5))); \
    prod = prod + (YN(2) * (YO(25) * RCT(1, 6))); \
    prod = prod + (YN(13) * (YN(10) * RCS(75))); \
    prod = prod + (YN(0) * (YO(25) * RCS(77))); \
    prod = prod + (YN(11) * (YN(10) * RCS(79))); \
    prod = prod + (YN(5) * (YO(25) * RCS(81))); \
    prod = prod + (YN(11) * ((YN(8) * YN(4)) * RCS(83))); \
    prod = prod + (YN(18) * ((YN(8) * YN(2)) * RCS(85))); \
    prod = prod + (YN(11) * ((YN(10) * YN(4)) * RCS(87))); \
    prod = prod + (YN(1) * (YO(31) * RCS(89))); \
    prod = prod + (YN(13) * (YN(8) * RCT(1, 7))); \
    prod = prod + (YN(4) * (YO(31) * RCS(92))); \
    prod = prod + (YN(3) * (YO(31) * RCS(96))); \
    prod = prod + (YN(2) * (YO(31) * RCS(100))); \
    prod = prod + (YN(13) * (YO(31) * RCS(104))); \
    prod = prod + (YN(6) * (YO(31) * RCS(108))); \
    extra = 0.0; \
    rhs1 = rho * Y0(23) + dt * WM(23) * (prod + extra); \
    loss = (YN(2) * RCT(1, 8)); \
    loss = loss + (YN(3) * RCT(1, 9)); \
    loss = loss + RCT(1, 10); \
    loss = loss + (YN(2) * RCS(74)); \
    loss = loss + (YN(2) * RCS(76)); \
    loss = loss + (YN(3) * RCS(78)); \
    loss = loss + (YN(4) * RCS(80)); \
    loss = loss + (YN(1) * RCS(82)); \
    loss = loss + (YN(13) * RCS(84)); \
    loss = loss + (YN(6) * RCS(86)); \
    loss = loss + (YN(6) * RCS(88)); \
    loss = loss + RCT(1, 11); \
    loss = loss + (YN(5) * RCS(93)); \
    loss = loss + (YN(4) * RCS(97)); \
    loss = loss + (YN(0) * RCS(101)); \
    loss = loss + (YN(12) * RCS(105)); \
    loss = loss + (YN(7) * RCS(109)); \
    rhs2 = -(dt * WM(23) * loss); \
    ppp = rho - FACE_SUM(23); \
    fnew = sor2 * YO(23) + (rhs1 - FACE_NBR(23)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(23) - fnew); \
    UC_UPDATE_TAIL(23); \
    TM_WAIT(0); \
    TM_LD(1, 0, 418); \
    TM_LD(1, 1, 412); \
    TM_LD(1, 2, 416); \
    TM_LD(1, 3, 406); \
    TM_LD(1, 4, 424); \
    TM_LD(1, 5, 432); \
    TM_LD(1, 6, 404); \
    TM_LD(1, 7, 426); \
    TM_LD(1, 8, 434); \
    TM_LD(1, 9, 420); \
    TM_LD(1, 10, 422); \
    TM_LD(1, 11, 410); \
    prod = (YN(16) * (YN(6) * RCT(0, 0))); \
    prod = prod + (YN(13) * ((YN(8) * YN(7)) * RCS(9))); \
    extra = 0.0; \
    rhs1 = rho * Y0(24) + dt * WM(24) * (prod + extra); \
    loss = (YN(4) * RCT(0, 1)); \
    loss = loss + (YN(6) * RCS(8)); \
    rhs2 = -(dt * WM(24) * loss); \
    ppp = rho - FACE_SUM(24); \
    fnew = sor2 * YO(24) + (rhs1 - FACE_NBR(24)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(24) - fnew); \
    UC_UPDATE_TAIL(24); \
    prod = (YN(21) * (YN(4) * RCS(18))); \
    prod = prod + (YN(13) * (YN(8) * RCS(23))); \
    prod = prod + (YN(14) * (YN(9) * RCS(25))); \
    prod = prod + (YN(4) * (YO(26) * RCS(27))); \
    prod = prod + (YN(18) * (YN(8) * RCS(29))); \
    prod = prod + (YN(8) * (YO(28) * RCS(59))); \
    prod = prod + (YN(23) * RCT(0, 2)); \
    prod = prod + (YN(23) * (YN(2) * RCS(76))); \
    prod = prod + (YN(23) * (YN(4) * RCS(80))); \
    prod = prod + (YN(1) * (YO(37) * RCS(176))); \
    prod = prod + (YN(3) * (YO(39) * RCS(196))); \
    extra = 0.0; \
    rhs1 = rho * Y0(25) + dt * WM(25) * (prod + extra); \
    loss = (YN(2) * RCS(19)); \
    loss = loss + (YN(2) * RCS(22)); \
    loss = loss + (YN(3) * RCS(24)); \
    loss = loss + (YN(3) * RCS(26)); \
    loss = loss + (YN(13) * RCS(28)); \
    loss = loss + (YN(4) * RCS(58)); \
    loss = loss + (YN(2) * RCT(0, 3)); \
    loss = loss + (YN(0) * RCS(77)); \
    loss = loss + (YN(5) * RCS(81)); \
    loss = loss + (YN(10) * RCS(177)); \
    loss = loss + ((YN(13) * YN(2)) * RCS(197)); \
    rhs2 = -(dt * WM(25) * loss); \
    ppp = rho - FACE_SUM(25); \
    fnew = sor2 * YO(25) + (rhs1 - FACE_NBR(25)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(25) - fnew); \
    UC_UPDATE_TAIL(25); \
    prod = (YN(21) * (YN(3) * RCS(12))); \
    prod = prod + (YN(25) * (YN(3) * RCS(26))); \
    prod = prod + (YN(15) * (YN(8) * RCS(31))); \
    prod = prod + (YN(10) * ((YN(8) * YN(2)) * RCS(33))); \
    prod = prod + (YN(8) * ((YOS(6) * YN(2)) * RCS(35))); \
    prod = prod + (YN(8) * ((YOS(6) * YN(4)) * RCS(37))); \
    prod = prod + (YN(9) * ((YN(8) * YN(2)) * RCS(39))); \
    prod = prod + (YN(4) * (YO(27) * RCS(40))); \
    prod = prod + (YN(1) * (YO(27) * RCS(44))); \
    prod = prod + (YN(3) * (YO(36) * RCS(170))); \
    extra = 0.0; \
    rhs1 = rho * Y0(26) + dt * WM(26) * (prod + extra); \
    loss = (YN(2) * RCS(13)); \
    loss = loss + (YN(4) * RCS(27)); \
    loss = loss + (YN(2) * RCS(30)); \
    loss = loss + (YN(4) * RCS(32)); \
    loss = loss + (YN(3) * RCS(34)); \
    loss = loss + (YN(1) * RCS(36)); \
    loss = loss + (YN(1) * RCS(38)); \
    loss = loss + (YN(2) * RCS(41)); \
    loss = loss + (YN(3) * RCS(45)); \
    loss = loss + (YN(13) * RCS(171)); \
    rhs2 = -(dt * WM(26) * loss); \
    ppp = rho - FACE_SUM(26); \
    fnew = sor2 * YO(26) + (rhs1 - FACE_NBR(26)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(26) - fnew); \
    UC_UPDATE_TAIL(26); \
    prod = (YN(21) * (YN(4) * RCS(20))); \
    prod = prod + (YN(26) * (YN(2) * RCS(41))); \
    prod = prod + (YN(20) * (YN(8) * RCS(43))); \
    prod = prod + (YN(26) * (YN(3) * RCS(45))); \
    prod = prod + (YN(20) * (YN(9) * RCS(47))); \
    prod = prod + (YN(10) * (YN(8) * RCS(49))); \
    extra = 0.0; \
    rhs1 = rho * Y0(27) + dt * WM(27) * (prod + extra); \
    loss = (YN(5) * RCS(21)); \
    loss = loss + (YN(4) * RCS(40)); \
    loss = loss + (YN(3) * RCS(42)); \
    loss = loss + (YN(1) * RCS(44)); \
    loss = loss + (YN(1) * RCS(46)); \
    loss = loss + (YN(1) * RCS(48)); \
    rhs2 = -(dt * WM(27) * loss); \
    ppp = rho - FACE_SUM(27); \
    fnew = sor2 * YO(27) + (rhs1 - FACE_NBR(27)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(27) - fnew); \
    UC_UPDATE_TAIL(27); \
    prod = (YN(11) * (YN(0) * RCS(51))); \
    prod = prod + (YN(13) * (YN(4) * RCS(53))); \
    prod = prod + (YN(11) * (YN(5) * RCS(55))); \
    prod = prod + (YN(11) * (YN(6) * RCS(57))); \
    prod = prod + (YN(11) * (YN(2) * RCT(0, 4))); \
    prod = prod + (YN(17) * RCT(0, 5)); \
    prod = prod + (YN(25) * (YN(4) * RCS(58))); \
    prod = prod + (YN(4) * (YO(29) * RCS(60))); \
    prod = prod + (YN(2) * (YO(29) * RCS(64))); \
    prod = prod + (YN(3) * (YO(29) * RCS(68))); \
    prod = prod + (YN(6) * (YO(29) * RCS(70))); \
    prod = prod + (YN(1) * (YO(29) * RCS(72))); \
    prod = prod + (YO(30) * RCT(0, 6)); \
    prod = prod + (YN(2) * (YO(35) * RCS(148))); \
    prod = prod + (YN(2) * (YO(32) * RCS(160))); \
    extra = 0.0; \
    rhs1 = rho * Y0(28) + dt * WM(28) * (prod + extra); \
    loss = (YN(2) * RCS(50)); \
    loss = loss + (YN(2) * RCS(52)); \
    loss = loss + (YN(4) * RCS(54)); \
    loss = loss + (YN(1) * RCS(56)); \
    loss = loss + RCT(0, 7); \
    loss = loss + RCT(0, 8); \
    loss = loss + (YN(8) * RCS(59)); \
    loss = loss + (YN(5) * RCS(61)); \
    loss = loss + (YN(0) * RCS(65)); \
    loss = loss + (YN(4) * RCS(69)); \
    loss = loss + (YN(7) * RCS(71)); \
    loss = loss + (YN(6) * RCS(73)); \
    loss = loss + (YN(13) * RCT(0, 9)); \
    loss = loss + (YN(13) * RCS(149)); \
    loss = loss + (YN(13) * RCS(161)); \
    rhs2 = -(dt * WM(28) * loss); \
    ppp = rho - FACE_SUM(28); \
    fnew = sor2 * YO(28) + (rhs1 - FACE_NBR(28)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(28) - fnew); \
    UC_UPDATE_TAIL(28); \
    prod = (YN(28) * (YN(5) * RCS(61))); \
    prod = prod + (YN(17) * (YN(5) * RCS(63))); \
    prod = prod + (YN(28) * (YN(0) * RCS(65))); \
    prod = prod + (YN(17) * (YN(0) * RCS(67))); \
    prod = prod + (YN(28) * (YN(4) * RCS(69))); \
    prod = prod + (YN(28) * (YN(7) * RCS(71))); \
    prod = prod + (YN(28) * (YN(6) * RCS(73))); \
    prod = prod + (YN(13) * (YN(4) * RCT(0, 10))); \
    extra = 0.0; \
    rhs1 = rho * Y0(29) + dt * WM(29) * (prod + extra); \
    loss = (YN(4) * RCS(60)); \
    loss = loss + (YN(4) * RCS(62)); \
    loss = loss + (YN(2) * RCS(64)); \
    loss = loss + (YN(2) * RCS(66)); \
    loss = loss + (YN(3) * RCS(68)); \
    loss = loss + (YN(6) * RCS(70)); \
    loss = loss + (YN(1) * RCS(72)); \
    loss = loss + RCT(0, 11); \
    rhs2 = -(dt * WM(29) * loss); \
    ppp = rho - FACE_SUM(29); \
    fnew = sor2 * YO(29) + (rhs1 - FACE_NBR(29)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(29) - fnew); \
    UC_UPDATE_TAIL(29); \
    prod = (YN(28) * (YN(13) * RCT(0, 9))); \
    TM_WAIT(1); \
    TM_LD(0, 0, 408); \
    TM_LD(0, 1, 426); \
    TM_LD(0, 2, 430); \
    TM_LD(0, 3, 424); \
    TM_LD(0, 4, 428); \
    TM_LD(0, 5, 436); \
    TM_LD(0, 6, 442); \
    TM_LD(0, 7, 492); \
    TM_LD(0, 8, 438); \
    TM_LD(0, 9, 440); \
    TM_LD(0, 10, 494); \
    TM_LD(0, 11, 486); \
    prod = prod + (YN(16) * (YN(5) * RCT(1, 0))); \
    prod = prod + (YN(5) * (YO(33) * RCS(113))); \
    prod = prod + (YN(5) * (YO(32) * RCS(115))); \
    prod = prod + (YN(5) * (YO(35) * RCS(117))); \
    prod = prod + (YN(0) * (YO(33) * RCS(119))); \
    prod = prod + (YN(0) * (YO(32) * RCS(121))); \
    prod = prod + (YN(0) * (YO(35) * RCS(123))); \
    prod = prod + (YN(4) * (YO(33) * RCS(125))); \
    prod = prod + (YN(4) * (YO(32) * RCS(127))); \
    prod = prod + (YN(4) * (YO(35) * RCS(129))); \
    prod = prod + (YN(12) * (YO(33) * RCS(131))); \
    prod = prod + (YN(12) * (YO(32) * RCS(133))); \
    prod = prod + (YN(12) * (YO(35) * RCS(135))); \
    prod = prod + (YN(7) * (YO(32) * RCS(137))); \
    prod = prod + (YN(7) * (YO(33) * RCS(139))); \
    prod = prod + (YN(7) * (YO(35) * RCS(141))); \
    extra = 0.0; \
    rhs1 = rho * Y0(30) + dt * WM(30) * (prod + extra); \
    loss = RCT(1, 1); \
    loss = loss + RCT(1, 2); \
    loss = loss + (YN(4) * RCS(112)); \
    loss = loss + (YN(4) * RCS(114)); \
    loss = loss + (YN(4) * RCS(116)); \
    loss = loss + (YN(2) * RCS(118)); \
    loss = loss + (YN(2) * RCS(120)); \
    loss = loss + (YN(2) * RCS(122)); \
    loss = loss + (YN(3) * RCS(124)); \
    loss = loss + (YN(3) * RCS(126)); \
    loss = loss + (YN(3) * RCS(128)); \
    loss = loss + (YN(13) * RCS(130)); \
    loss = loss + (YN(13) * RCS(132)); \
    loss = loss + (YN(13) * RCS(134)); \
    loss = loss + (YN(6) * RCS(136)); \
    loss = loss + (YN(6) * RCS(138)); \
    loss = loss + (YN(6) * RCS(140)); \
    rhs2 = -(dt * WM(30) * loss); \
    ppp = rho - FACE_SUM(30); \
    fnew = sor2 * YO(30) + (rhs1 - FACE_NBR(30)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(30) - fnew); \
    UC_UPDATE_TAIL(30); \
    prod = (YN(23) * (YN(6) * RCS(88))); \
    prod = prod + (YN(13) * (YN(10) * RCT(1, 3))); \
    prod = prod + (YN(5) * (YO(34) * RCS(91))); \
    prod = prod + (YN(23) * (YN(5) * RCS(93))); \
    prod = prod + (YN(4) * (YO(34) * RCS(95))); \
    prod = prod + (YN(23) * (YN(4) * RCS(97))); \
    prod = prod + (YN(0) * (YO(34) * RCS(99))); \
    prod = prod + (YN(23) * (YN(0) * RCS(101))); \
    prod = prod + (YN(12) * (YO(34) * RCS(103))); \
    prod = prod + (YN(23) * (YN(12) * RCS(105))); \
    prod = prod + (YN(7) * (YO(34) * RCS(107))); \
    prod = prod + (YN(23) * (YN(7) * RCS(109))); \
    prod = prod + (YN(6) * (YO(34) * RCS(111))); \
    prod = prod + (YO(35) * RCT(1, 4)); \
    prod = prod + (YN(1) * (YO(35) * RCS(144))); \
    prod = prod + (YN(4) * (YO(35) * RCS(152))); \
    prod = prod + (YN(1) * (YO(32) * RCS(154))); \
    prod = prod + (YN(3) * (YO(32) * RCS(156))); \
    prod = prod + (YN(6) * (YO(32) * RCS(162))); \
    prod = prod + (YN(4) * (YO(32) * RCS(164))); \
    prod = prod + (YO(32) * RCT(1, 5)); \
    extra = 0.0; \
    rhs1 = rho * Y0(31) + dt * WM(31) * (prod + extra); \
    loss = (YN(1) * RCS(89)); \
    loss = loss + RCT(1, 6); \
    loss = loss + (YN(4) * RCS(90)); \
    loss = loss + (YN(4) * RCS(92)); \
    loss = loss + (YN(3) * RCS(94)); \
    loss = loss + (YN(3) * RCS(96)); \
    loss = loss + (YN(2) * RCS(98)); \
    loss = loss + (YN(2) * RCS(100)); \
    loss = loss + (YN(13) * RCS(102)); \
    loss = loss + (YN(13) * RCS(104)); \
    loss = loss + (YN(6) * RCS(106)); \
    loss = loss + (YN(6) * RCS(108)); \
    loss = loss + (YN(1) * RCS(110)); \
    loss = loss + (YN(2) * RCT(1, 7)); \
    loss = loss + (YN(6) * RCS(145)); \
    loss = loss + (YN(5) * RCS(153)); \
    loss = loss + (YN(6) * RCS(155)); \
    loss = loss + (YN(4) * RCS(157)); \
    loss = loss + ((YN(4) * YN(4)) * RCS(163)); \
    loss = loss + (YN(5) * RCS(165)); \
    loss = loss + (YN(2) * RCT(1, 8)); \
    rhs2 = -(dt * WM(31) * loss); \
    ppp = rho - FACE_SUM(31); \
    fnew = sor2 * YO(31) + (rhs1 - FACE_NBR(31)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(31) - fnew); \
    UC_UPDATE_TAIL(31); \
    prod = (YN(30) * (YN(4) * RCS(114))); \
    prod = prod + (YN(30) * (YN(2) * RCS(120))); \
    prod = prod + (YN(30) * (YN(3) * RCS(126))); \
    prod = prod + (YN(30) * (YN(13) * RCS(132))); \
    prod = prod + (YN(30) * (YN(6) * RCS(136))); \
    prod = prod + (YN(31) * (YN(6) * RCS(155))); \
    prod = prod + (YN(31) * (YN(4) * RCS(157))); \
    prod = prod + (YN(16) * (YN(5) * RCS(159))); \
    prod = prod + (YN(28) * (YN(13) * RCS(161))); \
    prod = prod + (YN(31) * ((YN(4) * YN(4)) * RCS(163))); \
    prod = prod + (YN(31) * (YN(5) * RCS(165))); \
    prod = prod + (YN(31) * (YN(2) * RCT(1, 8))); \
    extra = 0.0; \
    rhs1 = rho * Y0(32) + dt * WM(32) * (prod + extra); \
    loss = (YN(5) * RCS(115)); \
    loss = loss + (YN(0) * RCS(121)); \
    loss = loss + (YN(4) * RCS(127)); \
    loss = loss + (YN(12) * RCS(133)); \
    loss = loss + (YN(7) * RCS(137)); \
    loss = loss + (YN(1) * RCS(154)); \
    loss = loss + (YN(3) * RCS(156)); \
    loss = loss + (YN(2) * RCS(158)); \
    loss = loss + (YN(2) * RCS(160)); \
    loss = loss + (YN(6) * RCS(162)); \
    loss = loss + (YN(4) * RCS(164)); \
    loss = loss + RCT(1, 5); \
    rhs2 = -(dt * WM(32) * loss); \
    ppp = rho - FACE_SUM(32); \
    fnew = sor2 * YO(32) + (rhs1 - FACE_NBR(32)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(32) - fnew); \
    UC_UPDATE_TAIL(32); \
    prod = (YN(30) * (YN(4) * RCS(112))); \
    prod = prod + (YN(30) * (YN(2) * RCS(118))); \
    prod = prod + (YN(30) * (YN(3) * RCS(124))); \
    prod = prod + (YN(30) * (YN(13) * RCS(130))); \
    prod = prod + (YN(30) * (YN(6) * RCS(138))); \
    prod = prod + (YN(16) * (YN(4) * RCT(1, 9))); \
    extra = 0.0; \
    rhs1 = rho * Y0(33) + dt * WM(33) * (prod + extra); \
    loss = (YN(5) * RCS(113)); \
    loss = loss + (YN(0) * RCS(119)); \
    loss = loss + (YN(4) * RCS(125)); \
    loss = loss + (YN(12) * RCS(131)); \
    loss = loss + (YN(7) * RCS(139)); \
    loss = loss + RCT(1, 10); \
    rhs2 = -(dt * WM(33) * loss); \
    ppp = rho - FACE_SUM(33); \
    fnew = sor2 * YO(33) + (rhs1 - FACE_NBR(33)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(33) - fnew); \
    UC_UPDATE_TAIL(33); \
    prod = (YN(13) * (YN(8) * RCT(1, 11))); \
    prod = prod + (YN(31) * (YN(4) * RCS(90))); \
    prod = prod + (YN(31) * (YN(3) * RCS(94))); \
    prod = prod + (YN(31) * (YN(2) * RCS(98))); \
    prod = prod + (YN(31) * (YN(13) * RCS(102))); \
    prod = prod + (YN(31) * (YN(6) * RCS(106))); \
    prod = prod + (YN(31) * (YN(1) * RCS(110))); \
    extra = 0.0; \
    rhs1 = rho * Y0(34) + dt * WM(34) * (prod + extra); \
    TM_WAIT(0); \
    TM_LD(1, 0, 484); \
    TM_LD(1, 1, 440); \
    TM_LD(1, 2, 444); \
    TM_LD(1, 3, 450); \
    TM_LD(1, 4, 496); \
    TM_LD(1, 5, 500); \
    TM_LD(1, 6, 508); \
    TM_LD(1, 7, 442); \
    TM_LD(1, 8, 446); \
    TM_LD(1, 9, 448); \
    TM_LD(1, 10, 498); \
    TM_LD(1, 11, 502); \
    loss = RCT(0, 0); \
    loss = loss + (YN(5) * RCS(91)); \
    loss = loss + (YN(4) * RCS(95)); \
    loss = loss + (YN(0) * RCS(99)); \
    loss = loss + (YN(12) * RCS(103)); \
    loss = loss + (YN(7) * RCS(107)); \
    loss = loss + (YN(6) * RCS(111)); \
    rhs2 = -(dt * WM(34) * loss); \
    ppp = rho - FACE_SUM(34); \
    fnew = sor2 * YO(34) + (rhs1 - FACE_NBR(34)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(34) - fnew); \
    UC_UPDATE_TAIL(34); \
    prod = (YN(30) * (YN(4) * RCS(116))); \
    prod = prod + (YN(30) * (YN(2) * RCS(122))); \
    prod = prod + (YN(30) * (YN(3) * RCS(128))); \
    prod = prod + (YN(30) * (YN(13) * RCS(134))); \
    prod = prod + (YN(30) * (YN(6) * RCS(140))); \
    prod = prod + (YN(18) * (YN(6) * RCS(142))); \
    prod = prod + (YN(31) * (YN(2) * RCT(0, 1))); \
    prod = prod + (YN(13) * (YN(11) * RCT(0, 2))); \
    prod = prod + (YN(31) * (YN(6) * RCS(145))); \
    prod = prod + (YN(18) * (YN(9) * RCS(147))); \
    prod = prod + (YN(28) * (YN(13) * RCS(149))); \
    prod = prod + (YN(16) * (YN(5) * RCS(151))); \
    prod = prod + (YN(31) * (YN(5) * RCS(153))); \
    extra = 0.0; \
    rhs1 = rho * Y0(35) + dt * WM(35) * (prod + extra); \
    loss = (YN(5) * RCS(117)); \
    loss = loss + (YN(0) * RCS(123)); \
    loss = loss + (YN(4) * RCS(129)); \
    loss = loss + (YN(12) * RCS(135)); \
    loss = loss + (YN(7) * RCS(141)); \
    loss = loss + (YN(4) * RCS(143)); \
    loss = loss + RCT(0, 3); \
    loss = loss + RCT(0, 4); \
    loss = loss + (YN(1) * RCS(144)); \
    loss = loss + (YN(8) * RCS(146)); \
    loss = loss + (YN(2) * RCS(148)); \
    loss = loss + (YN(2) * RCS(150)); \
    loss = loss + (YN(4) * RCS(152)); \
    rhs2 = -(dt * WM(35) * loss); \
    ppp = rho - FACE_SUM(35); \
    fnew = sor2 * YO(35) + (rhs1 - FACE_NBR(35)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(35) - fnew); \
    UC_UPDATE_TAIL(35); \
    prod = (YN(16) * (YN(8) * RCS(167))); \
    prod = prod + (YN(21) * (YN(13) * RCS(168))); \
    prod = prod + (YN(26) * (YN(13) * RCS(171))); \
    prod = prod + (YN(2) * (YO(37) * RCT(0, 5))); \
    prod = prod + (YN(6) * (YO(37) * RCS(172))); \
    prod = prod + (YN(5) * (YO(37) * RCS(175))); \
    prod = prod + (YO(38) * RCT(0, 6)); \
    prod = prod + (YN(2) * (YO(38) * RCS(178))); \
    prod = prod + (YN(1) * (YO(38) * RCS(180))); \
    prod = prod + (YN(13) * (YO(38) * RCS(182))); \
    prod = prod + (YN(4) * (YO(38) * RCS(184))); \
    prod = prod + (YN(10) * (YO(37) * RCS(186))); \
    prod = prod + (YN(13) * ((YN(10) * YN(8)) * RCS(191))); \
    prod = prod + (YO(45) * RCT(0, 7)); \
    prod = prod + (YN(1) * (YO(45) * RCS(244))); \
    prod = prod + (YN(6) * (YO(45) * RCS(248))); \
    extra = 0.0; \
    rhs1 = rho * Y0(36) + dt * WM(36) * (prod + extra); \
    loss = (YN(3) * RCS(166)); \
    loss = loss + (YN(2) * RCS(169)); \
    loss = loss + (YN(3) * RCS(170)); \
    loss = loss + RCT(0, 8); \
    loss = loss + (YN(1) * RCS(173)); \
    loss = loss + (YN(4) * RCS(174)); \
    loss = loss + (YN(2) * RCT(0, 9)); \
    loss = loss + (YN(0) * RCS(179)); \
    loss = loss + (YN(6) * RCS(181)); \
    loss = loss + (YN(12) * RCS(183)); \
    loss = loss + (YN(5) * RCS(185)); \
    loss = loss + (YN(8) * RCS(187)); \
    loss = loss + (YN(1) * RCS(190)); \
    loss = loss + (YN(16) * RCT(0, 10)); \
    loss = loss + ((YN(22) * YN(6)) * RCS(245)); \
    loss = loss + ((YN(22) * YN(7)) * RCS(249)); \
    rhs2 = -(dt * WM(36) * loss); \
    ppp = rho - FACE_SUM(36); \
    fnew = sor2 * YO(36) + (rhs1 - FACE_NBR(36)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(36) - fnew); \
    UC_UPDATE_TAIL(36); \
    prod = (YN(36) * RCT(0, 8)); \
    prod = prod + (YN(36) * (YN(1) * RCS(173))); \
    prod = prod + (YN(36) * (YN(4) * RCS(174))); \
    prod = prod + (YN(25) * (YN(10) * RCS(177))); \
    prod = prod + (YN(36) * (YN(8) * RCS(187))); \
    prod = prod + (YN(22) * ((YN(4) * YN(8)) * RCS(189))); \
    prod = prod + (YO(43) * RCT(0, 11)); \
    extra = 0.0; \
    rhs1 = rho * Y0(37) + dt * WM(37) * (prod + extra); \
    loss = (YN(2) * RCT(0, 5)); \
    loss = loss + (YN(6) * RCS(172)); \
    loss = loss + (YN(5) * RCS(175)); \
    loss = loss + (YN(1) * RCS(176)); \
    loss = loss + (YN(10) * RCS(186)); \
    loss = loss + (YN(6) * RCS(188)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 510); \
    TM_LD(0, 1, 448); \
    TM_LD(0, 2, 452); \
    TM_LD(0, 3, 466); \
    TM_LD(0, 4, 474); \
    TM_LD(0, 5, 488); \
    TM_LD(0, 6, 504); \
    TM_LD(0, 7, 450); \
    TM_LD(0, 8, 454); \
    TM_LD(0, 9, 464); \
    TM_LD(0, 10, 472); \
    TM_LD(0, 11, 490); \
    loss = loss + (YN(13) * RCT(1, 0)); \
    rhs2 = -(dt * WM(37) * loss); \
    ppp = rho - FACE_SUM(37); \
    fnew = sor2 * YO(37) + (rhs1 - FACE_NBR(37)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(37) - fnew); \
    UC_UPDATE_TAIL(37); \
    prod = (YN(36) * (YN(2) * RCT(1, 1))); \
    prod = prod + (YN(36) * (YN(0) * RCS(179))); \
    prod = prod + (YN(36) * (YN(6) * RCS(181))); \
    prod = prod + (YN(36) * (YN(12) * RCS(183))); \
    prod = prod + (YN(21) * (YN(13) * RCT(1, 2))); \
    prod = prod + (YN(36) * (YN(5) * RCS(185))); \
    prod = prod + (YN(4) * (YO(39) * RCS(194))); \
    prod = prod + (YN(2) * (YO(39) * RCS(198))); \
    prod = prod + (YO(39) * RCT(1, 3)); \
    prod = prod + (YN(1) * (YO(39) * RCS(201))); \
    prod = prod + (YN(22) * ((YN(4) * YN(11)) * RCS(203))); \
    prod = prod + (YN(22) * (YN(13) * RCS(206))); \
    prod = prod + (YN(4) * (YO(43) * RCS(238))); \
    prod = prod + (YO(45) * RCT(1, 4)); \
    prod = prod + (YN(1) * (YO(45) * RCS(242))); \
    prod = prod + (YN(6) * (YO(45) * RCS(246))); \
    prod = prod + (YO(48) * RCT(1, 5)); \
    prod = prod + (YN(2) * (YO(48) * RCS(269))); \
    prod = prod + (YO(47) * RCT(1, 6)); \
    extra = 0.0; \
    rhs1 = rho * Y0(38) + dt * WM(38) * (prod + extra); \
    loss = RCT(1, 7); \
    loss = loss + (YN(2) * RCS(178)); \
    loss = loss + (YN(1) * RCS(180)); \
    loss = loss + (YN(13) * RCS(182)); \
    loss = loss + RCT(1, 8); \
    loss = loss + (YN(4) * RCS(184)); \
    loss = loss + (YN(5) * RCS(195)); \
    loss = loss + (YN(0) * RCS(199)); \
    loss = loss + (YN(2) * RCT(1, 9)); \
    loss = loss + (YN(6) * RCS(200)); \
    loss = loss + (YN(6) * RCS(202)); \
    loss = loss + (YN(2) * RCS(207)); \
    loss = loss + ((YO(44) * YN(2)) * RCS(239)); \
    loss = loss + (YN(22) * RCT(1, 10)); \
    loss = loss + ((YN(21) * YN(6)) * RCS(243)); \
    loss = loss + ((YN(21) * YN(7)) * RCS(247)); \
    loss = loss + (YN(18) * RCT(1, 11)); \
    loss = loss + ((YN(0) * YN(16)) * RCS(270)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 506); \
    TM_LD(1, 1, 458); \
    TM_LD(1, 2, 456); \
    TM_LD(1, 3, 462); \
    TM_LD(1, 4, 464); \
    TM_LD(1, 5, 460); \
    TM_LD(1, 6, 466); \
    TM_LD(1, 7, 470); \
    TM_LD(1, 8, 472); \
    TM_LD(1, 9, 468); \
    TM_LD(1, 10, 474); \
    TM_LD(1, 11, 478); \
    loss = loss + (YN(13) * RCT(0, 0)); \
    rhs2 = -(dt * WM(38) * loss); \
    ppp = rho - FACE_SUM(38); \
    fnew = sor2 * YO(38) + (rhs1 - FACE_NBR(38)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(38) - fnew); \
    UC_UPDATE_TAIL(38); \
    prod = (YN(18) * (YN(10) * RCS(193))); \
    prod = prod + (YN(38) * (YN(5) * RCS(195))); \
    prod = prod + (YN(25) * ((YN(13) * YN(2)) * RCS(197))); \
    prod = prod + (YN(38) * (YN(0) * RCS(199))); \
    prod = prod + (YN(38) * (YN(2) * RCT(0, 1))); \
    prod = prod + (YN(38) * (YN(6) * RCS(200))); \
    prod = prod + (YN(22) * (YN(13) * RCT(0, 2))); \
    prod = prod + (YN(16) * (YN(13) * RCS(205))); \
    prod = prod + (YO(41) * RCT(0, 3)); \
    prod = prod + (YN(1) * (YO(41) * RCS(228))); \
    prod = prod + (YO(42) * RCT(0, 4)); \
    prod = prod + (YN(1) * (YO(42) * RCS(230))); \
    prod = prod + (YO(45) * RCT(0, 5)); \
    prod = prod + (YO(48) * RCT(0, 6)); \
    prod = prod + (YN(4) * (YO(48) * RCS(261))); \
    prod = prod + (YN(2) * (YO(48) * RCS(263))); \
    prod = prod + (YN(2) * (YO(48) * RCS(267))); \
    prod = prod + (YN(2) * (YO(47) * RCS(275))); \
    extra = (1.0 * (YN(2) * (YO(46) * RCS(251)))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(259)))); \
    rhs1 = rho * Y0(39) + dt * WM(39) * (prod + extra); \
    loss = (YN(3) * RCS(192)); \
    loss = loss + (YN(4) * RCS(194)); \
    loss = loss + (YN(3) * RCS(196)); \
    loss = loss + (YN(2) * RCS(198)); \
    loss = loss + RCT(0, 7); \
    loss = loss + (YN(1) * RCS(201)); \
    loss = loss + RCT(0, 8); \
    loss = loss + (YN(2) * RCS(204)); \
    loss = loss + (YN(2) * RCT(0, 9)); \
    loss = loss + (YN(6) * RCS(229)); \
    loss = loss + (YN(2) * RCT(0, 10)); \
    loss = loss + (YN(6) * RCS(231)); \
    loss = loss + (YN(21) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 480); \
    TM_LD(0, 1, 484); \
    TM_LD(0, 2, 476); \
    TM_LD(0, 3, 482); \
    TM_LD(0, 4, 486); \
    TM_LD(0, 5, 490); \
    TM_LD(0, 6, 494); \
    TM_LD(0, 7, 498); \
    TM_LD(0, 8, 488); \
    TM_LD(0, 9, 492); \
    TM_LD(0, 10, 496); \
    TM_LD(0, 11, 510); \
    loss = loss + (YN(16) * RCT(1, 0)); \
    loss = loss + ((YN(5) * YN(22)) * RCS(262)); \
    loss = loss + ((YN(0) * YN(22)) * RCS(264)); \
    loss = loss + (YN(18) * RCS(268)); \
    loss = loss + (YN(13) * RCS(276)); \
    rhs2 = -(dt * WM(39) * loss); \
    ppp = rho - FACE_SUM(39); \
    fnew = sor2 * YO(39) + (rhs1 - FACE_NBR(39)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(39) - fnew); \
    UC_UPDATE_TAIL(39); \
    prod = (YN(18) * (YN(13) * RCT(1, 1))); \
    prod = prod + (YN(6) * (YO(41) * RCS(209))); \
    prod = prod + (YN(6) * (YO(42) * RCS(211))); \
    prod = prod + (YN(0) * (YO(41) * RCS(213))); \
    prod = prod + (YN(0) * (YO(42) * RCS(215))); \
    prod = prod + (YN(4) * (YO(41) * RCS(217))); \
    prod = prod + (YN(4) * (YO(42) * RCS(219))); \
    prod = prod + (YN(5) * (YO(42) * RCS(221))); \
    prod = prod + (YN(5) * (YO(41) * RCS(223))); \
    prod = prod + (YN(7) * (YO(41) * RCS(225))); \
    prod = prod + (YN(7) * (YO(42) * RCS(227))); \
    extra = 0.0; \
    rhs1 = rho * Y0(40) + dt * WM(40) * (prod + extra); \
    loss = RCT(1, 2); \
    loss = loss + (YN(1) * RCS(208)); \
    loss = loss + (YN(1) * RCS(210)); \
    loss = loss + (YN(2) * RCS(212)); \
    loss = loss + (YN(2) * RCS(214)); \
    loss = loss + (YN(3) * RCS(216)); \
    loss = loss + (YN(3) * RCS(218)); \
    loss = loss + (YN(4) * RCS(220)); \
    loss = loss + (YN(4) * RCS(222)); \
    loss = loss + (YN(6) * RCS(224)); \
    loss = loss + (YN(6) * RCS(226)); \
    rhs2 = -(dt * WM(40) * loss); \
    ppp = rho - FACE_SUM(40); \
    fnew = sor2 * YO(40) + (rhs1 - FACE_NBR(40)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(40) - fnew); \
    UC_UPDATE_TAIL(40); \
    prod = (YN(40) * (YN(1) * RCS(208))); \
    prod = prod + (YN(40) * (YN(2) * RCS(212))); \
    prod = prod + (YN(40) * (YN(3) * RCS(216))); \
    prod = prod + (YN(40) * (YN(4) * RCS(222))); \
    prod = prod + (YN(40) * (YN(6) * RCS(224))); \
    prod = prod + (YO(42) * RCT(1, 3)); \
    prod = prod + (YN(39) * (YN(2) * RCT(1, 4))); \
    prod = prod + (YN(39) * (YN(6) * RCS(229))); \
    extra = 0.0; \
    rhs1 = rho * Y0(41) + dt * WM(41) * (prod + extra); \
    loss = (YN(6) * RCS(209)); \
    loss = loss + (YN(0) * RCS(213)); \
    loss = loss + (YN(4) * RCS(217)); \
    loss = loss + (YN(5) * RCS(223)); \
    loss = loss + (YN(7) * RCS(225)); \
    loss = loss + RCT(1, 5); \
    loss = loss + RCT(1, 6); \
    loss = loss + (YN(1) * RCS(228)); \
    rhs2 = -(dt * WM(41) * loss); \
    ppp = rho - FACE_SUM(41); \
    fnew = sor2 * YO(41) + (rhs1 - FACE_NBR(41)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(41) - fnew); \
    UC_UPDATE_TAIL(41); \
    prod = (YN(40) * (YN(1) * RCS(210))); \
    prod = prod + (YN(40) * (YN(2) * RCS(214))); \
    prod = prod + (YN(40) * (YN(3) * RCS(218))); \
    prod = prod + (YN(40) * (YN(4) * RCS(220))); \
    prod = prod + (YN(40) * (YN(6) * RCS(226))); \
    prod = prod + (YN(41) * RCT(1, 5)); \
    prod = prod + (YN(16) * (YN(13) * RCT(1, 7))); \
    prod = prod + (YN(39) * (YN(2) * RCT(1, 8))); \
    prod = prod + (YN(39) * (YN(6) * RCS(231))); \
    extra = 0.0; \
    rhs1 = rho * Y0(42) + dt * WM(42) * (prod + extra); \
    loss = (YN(6) * RCS(211)); \
    loss = loss + (YN(0) * RCS(215)); \
    loss = loss + (YN(4) * RCS(219)); \
    loss = loss + (YN(5) * RCS(221)); \
    loss = loss + (YN(7) * RCS(227)); \
    loss = loss + RCT(1, 3); \
    loss = loss + RCT(1, 9); \
    loss = loss + RCT(1, 10); \
    loss = loss + (YN(1) * RCS(230)); \
    rhs2 = -(dt * WM(42) * loss); \
    ppp = rho - FACE_SUM(42); \
    fnew = sor2 * YO(42) + (rhs1 - FACE_NBR(42)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(42) - fnew); \
    UC_UPDATE_TAIL(42); \
    prod = (YN(22) * ((YN(21) * YN(2)) * RCS(233))); \
    prod = prod + (YN(22) * (YOS(7) * RCT(1, 11))); \
    TM_WAIT(0); \
    TM_LD(1, 0, 508); \
    TM_LD(1, 1, 502); \
    TM_LD(1, 2, 506); \
    TM_LD(1, 3, 500); \
    TM_LD(1, 4, 504); \
    prod = prod + (YN(22) * (YOS(7) * RCT(0, 0))); \
    prod = prod + (YN(22) * (YN(16) * RCS(235))); \
    prod = prod + (YN(22) * ((YN(0) * YN(21)) * RCS(237))); \
    prod = prod + (YN(38) * ((YO(44) * YN(2)) * RCS(239))); \
    prod = prod + (YN(22) * ((YN(12) * YN(21)) * RCS(241))); \
    prod = prod + (YN(37) * (YN(13) * RCT(0, 1))); \
    prod = prod + (YN(2) * (YO(48) * RCS(271))); \
    prod = prod + (YN(4) * (YO(47) * RCS(279))); \
    extra = 0.0; \
    rhs1 = rho * Y0(43) + dt * WM(43) * (prod + extra); \
    loss = RCS(232); \
    loss = loss + RCT(0, 2); \
    loss = loss + RCT(0, 3); \
    loss = loss + (YN(2) * RCS(234)); \
    loss = loss + (YN(2) * RCS(236)); \
    loss = loss + (YN(4) * RCS(238)); \
    loss = loss + (YN(13) * RCS(240)); \
    loss = loss + RCT(0, 4); \
    loss = loss + ((YN(0) * YN(13)) * RCS(272)); \
    loss = loss + ((YN(5) * YN(2)) * RCS(280)); \
    rhs2 = -(dt * WM(43) * loss); \
    ppp = rho - FACE_SUM(43); \
    fnew = sor2 * YO(43) + (rhs1 - FACE_NBR(43)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(43) - fnew); \
    UC_UPDATE_TAIL(43); \
    prod = (YN(43) * (YN(4) * RCS(238))); \
    extra = 0.0; \
    rhs1 = rho * Y0(44) + dt * WM(44) * (prod + extra); \
    loss = ((YN(2) * YN(38)) * RCS(239)); \
    rhs2 = -(dt * WM(44) * loss); \
    ppp = rho - FACE_SUM(44); \
    fnew = sor2 * YO(44) + (rhs1 - FACE_NBR(44)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(44) - fnew); \
    UC_UPDATE_TAIL(44); \
    prod = (YN(39) * (YN(21) * RCT(0, 5))); \
    prod = prod + (YN(36) * (YN(16) * RCT(0, 6))); \
    prod = prod + (YN(38) * (YN(22) * RCT(0, 7))); \
    prod = prod + (YN(38) * ((YN(21) * YN(6)) * RCS(243))); \
    prod = prod + (YN(36) * ((YN(22) * YN(6)) * RCS(245))); \
    prod = prod + (YN(38) * ((YN(21) * YN(7)) * RCS(247))); \
    prod = prod + (YN(36) * ((YN(22) * YN(7)) * RCS(249))); \
    extra = 0.0; \
    rhs1 = rho * Y0(45) + dt * WM(45) * (prod + extra); \
    loss = RCT(0, 8); \
    loss = loss + RCT(0, 9); \
    loss = loss + RCT(0, 10); \
    loss = loss + (YN(1) * RCS(242)); \
    loss = loss + (YN(1) * RCS(244)); \
    loss = loss + (YN(6) * RCS(246)); \
    loss = loss + (YN(6) * RCS(248)); \
    rhs2 = -(dt * WM(45) * loss); \
    ppp = rho - FACE_SUM(45); \
    fnew = sor2 * YO(45) + (rhs1 - FACE_NBR(45)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(45) - fnew); \
    UC_UPDATE_TAIL(45); \
    prod = 0.0; \
    prod = prod + 0.0; \
    prod = prod + 0.0; \
    prod = prod + 0.0; \
    prod = prod + (YN(18) * ((YN(0) * YO(48)) * RCS(255))); \
    prod = prod + (YN(18) * ((YN(5) * YO(48)) * RCS(257))); \
    prod = prod + 0.0; \
    prod = prod + 0.0; \
    prod = prod + 0.0; \
    extra = 0.0; \
    rhs1 = rho * Y0(46) + dt * WM(46) * (prod + extra); \
    loss = RCS(250); \
    loss = loss + (YN(2) * RCS(251)); \
    loss = loss + (YN(2) * RCS(252)); \
    loss = loss + (YN(2) * RCS(253)); \
    loss = loss + (YN(2) * RCS(254)); \
    loss = loss + (YN(4) * RCS(256)); \
    loss = loss + (YN(4) * RCS(258)); \
    loss = loss + (YN(4) * RCS(259)); \
    loss = loss + (YN(4) * RCS(260)); \
    rhs2 = -(dt * WM(46) * loss); \
    ppp = rho - FACE_SUM(46); \
    fnew = sor2 * YO(46) + (rhs1 - FACE_NBR(46)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(46) - fnew); \
    UC_UPDATE_TAIL(46); \
    prod = (YN(38) * (YN(13) * RCT(0, 11))); \
    prod = prod + (YN(18) * (YN(16) * RCS(274))); \
    prod = prod + (YN(39) * (YN(13) * RCS(276))); \
    prod = prod + (YN(22) * ((YN(0) * YN(16)) * RCS(278))); \
    prod = prod + (YN(43) * ((YN(5) * YN(2)) * RCS(280))); \
    extra = (1.0 * (YN(46) * (YN(2) * RCS(252)))); \
    extra = extra + (1.0 * (YN(46) * (YN(4) * RCS(258)))); \
    rhs1 = rho * Y0(47) + dt * WM(47) * (prod + extra); \
    TM_WAIT(1); \
    loss = RCT(1, 0); \
    loss = loss + (YN(2) * RCS(273)); \
    loss = loss + (YN(2) * RCS(275)); \
    loss = loss + (YN(2) * RCS(277)); \
    loss = loss + (YN(4) * RCS(279)); \
    rhs2 = -(dt * WM(47) * loss); \
    ppp = rho - FACE_SUM(47); \
    fnew = sor2 * YO(47) + (rhs1 - FACE_NBR(47)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(47) - fnew); \
    UC_UPDATE_TAIL(47); \
    prod = (YN(46) * (YN(2) * RCS(254))); \
    prod = prod + (YN(46) * (YN(4) * RCS(256))); \
    prod = prod + (YN(38) * (YN(18) * RCT(1, 1))); \
    prod = prod + (YN(39) * (YN(16) * RCT(1, 2))); \
    prod = prod + (YN(39) * ((YN(5) * YN(22)) * RCS(262))); \
    prod = prod + (YN(39) * ((YN(0) * YN(22)) * RCS(264))); \
    prod = prod + (YN(16) * ((YOS(4) * YN(13)) * RCS(266))); \
    prod = prod + (YN(39) * (YN(18) * RCS(268))); \
    prod = prod + (YN(38) * ((YN(0) * YN(16)) * RCS(270))); \
    prod = prod + (YN(43) * ((YN(0) * YN(13)) * RCS(272))); \
    extra = 0.0; \
    rhs1 = rho * Y0(48) + dt * WM(48) * (prod + extra); \
    loss = ((YN(0) * YN(18)) * RCS(255)); \
    loss = loss + ((YN(5) * YN(18)) * RCS(257)); \
    loss = loss + RCT(1, 3); \
    loss = loss + RCT(1, 4); \
    loss = loss + (YN(4) * RCS(261)); \
    loss = loss + (YN(2) * RCS(263)); \
    loss = loss + (YN(2) * RCS(265)); \
    loss = loss + (YN(2) * RCS(267)); \
    loss = loss + (YN(2) * RCS(269)); \
    loss = loss + (YN(2) * RCS(271)); \
    rhs2 = -(dt * WM(48) * loss); \
    ppp = rho - FACE_SUM(48); \
    fnew = sor2 * YO(48) + (rhs1 - FACE_NBR(48)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(48) - fnew); \
    UC_UPDATE_TAIL(48); \
    extra = 0.0; \
    rhs1 = rho * Y0(49) + dt * WM(49) * (prod + extra); \
    rhs2 = 0.0; \
    ppp = rho - FACE_SUM(49); \
    fnew = sor2 * YO(49) + (rhs1 - FACE_NBR(49)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(49) - fnew); \
    UC_UPDATE_TAIL(49); \
    extra = 0.0; \
    rhs1 = rho * Y0(50) + dt * WM(50) * (prod + extra); \
    rhs2 = 0.0; \
    ppp = rho - FACE_SUM(50); \
    fnew = sor2 * YO(50) + (rhs1 - FACE_NBR(50)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(50) - fnew); \
    UC_UPDATE_TAIL(50); \
} while (0)
#ifdef __CUDACC__
static __constant__ int16_t uc_tr_trow[256] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51, 52, 53, 54, 55, 56, 57, 58, 59, 60, 61, 62, 63, 64, 65, 66, 67, 68, 69, 70, 71, 72, 73, 74, 75, 76, 77, 78, 79, 80, 81, 82, 83, 84, 85, 86, 87, 88, 89, 90, 91, 92, 93, 94, 95, 96, 97, 98, 99, 100, 101, 102, 103, 104, 105, 106, 107, 108, 109, 112, 113, 114, 115, 116, 117, 118, 119, 120, 121, 124, 125, 126, 127, 132, 133, 134, 135, 136, 137, 138, 139, 140, 141, 142, 143, 144, 145, 146, 147, 148, 149, 150, 151, 152, 153, 154, 155, 156, 157, 158, 159, 160, 161, 162, 163, 164, 165, 166, 167, 168, 169, 170, 171, 172, 173, 174, 175, 176, 177, 178, 179, 180, 181, 182, 183, 184, 185, 186, 187, 190, 191, 192, 193, 194, 195, 196, 197, 198, 199, 200, 201, 250, 251, 252, 253, 270, 271, 272, 273, 290, 291, 292, 293, 294, 295, 318, 319, 320, 321, 352, 353, 356, 357, 358, 359, 382, 383, 390, 391, 398, 399, 406, 407, 424, 425, 430, 431, 436, 437, 458, 459, 460, 461, 464, 465, 466, 467, 472, 473, 474, 475, 484, 485, 486, 487, 488, 489, 490, 491, 518, 519, 520, 521, 534, 535};
static __constant__ int16_t uc_tr_srow[281] = {110, 111, 122, 123, 128, 129, 130, 131, 188, 189, 202, 203, 204, 205, 206, 207, 208, 209, 210, 211, 212, 213, 214, 215, 216, 217, 218, 219, 220, 221, 222, 223, 224, 225, 226, 227, 228, 229, 230, 231, 232, 233, 234, 235, 236, 237, 238, 239, 240, 241, 242, 243, 244, 245, 246, 247, 248, 249, 254, 255, 256, 257, 258, 259, 260, 261, 262, 263, 264, 265, 266, 267, 268, 269, 274, 275, 276, 277, 278, 279, 280, 281, 282, 283, 284, 285, 286, 287, 288, 289, 296, 297, 298, 299, 300, 301, 302, 303, 304, 305, 306, 307, 308, 309, 310, 311, 312, 313, 314, 315, 316, 317, 322, 323, 324, 325, 326, 327, 328, 329, 330, 331, 332, 333, 334, 335, 336, 337, 338, 339, 340, 341, 342, 343, 344, 345, 346, 347, 348, 349, 350, 351, 354, 355, 360, 361, 362, 363, 364, 365, 366, 367, 368, 369, 370, 371, 372, 373, 374, 375, 376, 377, 378, 379, 380, 381, 384, 385, 386, 387, 388, 389, 392, 393, 394, 395, 396, 397, 400, 401, 402, 403, 404, 405, 408, 409, 410, 411, 412, 413, 414, 415, 416, 417, 418, 419, 420, 421, 422, 423, 426, 427, 428, 429, 432, 433, 434, 435, 438, 439, 440, 441, 442, 443, 444, 445, 446, 447, 448, 449, 450, 451, 452, 453, 454, 455, 456, 457, 462, 463, 468, 469, 470, 471, 476, 477, 478, 479, 480, 481, 482, 483, 492, 493, 494, 495, 496, 497, 498, 499, 500, 502, 504, 506, 508, 509, 510, 511, 512, 514, 516, 522, 523, 524, 525, 526, 527, 528, 529, 530, 531, 532, 533, 536, 537, 538, 539, 540, 541, 542, 543};
#else
static const short uc_tr_trow[256] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51, 52, 53, 54, 55, 56, 57, 58, 59, 60, 61, 62, 63, 64, 65, 66, 67, 68, 69, 70, 71, 72, 73, 74, 75, 76, 77, 78, 79, 80, 81, 82, 83, 84, 85, 86, 87, 88, 89, 90, 91, 92, 93, 94, 95, 96, 97, 98, 99, 100, 101, 102, 103, 104, 105, 106, 107, 108, 109, 112, 113, 114, 115, 116, 117, 118, 119, 120, 121, 124, 125, 126, 127, 132, 133, 134, 135, 136, 137, 138, 139, 140, 141, 142, 143, 144, 145, 146, 147, 148, 149, 150, 151, 152, 153, 154, 155, 156, 157, 158, 159, 160, 161, 162, 163, 164, 165, 166, 167, 168, 169, 170, 171, 172, 173, 174, 175, 176, 177, 178, 179, 180, 181, 182, 183, 184, 185, 186, 187, 190, 191, 192, 193, 194, 195, 196, 197, 198, 199, 200, 201, 250, 251, 252, 253, 270, 271, 272, 273, 290, 291, 292, 293, 294, 295, 318, 319, 320, 321, 352, 353, 356, 357, 358, 359, 382, 383, 390, 391, 398, 399, 406, 407, 424, 425, 430, 431, 436, 437, 458, 459, 460, 461, 464, 465, 466, 467, 472, 473, 474, 475, 484, 485, 486, 487, 488, 489, 490, 491, 518, 519, 520, 521, 534, 535};
static const short uc_tr_srow[281] = {110, 111, 122, 123, 128, 129, 130, 131, 188, 189, 202, 203, 204, 205, 206, 207, 208, 209, 210, 211, 212, 213, 214, 215, 216, 217, 218, 219, 220, 221, 222, 223, 224, 225, 226, 227, 228, 229, 230, 231, 232, 233, 234, 235, 236, 237, 238, 239, 240, 241, 242, 243, 244, 245, 246, 247, 248, 249, 254, 255, 256, 257, 258, 259, 260, 261, 262, 263, 264, 265, 266, 267, 268, 269, 274, 275, 276, 277, 278, 279, 280, 281, 282, 283, 284, 285, 286, 287, 288, 289, 296, 297, 298, 299, 300, 301, 302, 303, 304, 305, 306, 307, 308, 309, 310, 311, 312, 313, 314, 315, 316, 317, 322, 323, 324, 325, 326, 327, 328, 329, 330, 331, 332, 333, 334, 335, 336, 337, 338, 339, 340, 341, 342, 343, 344, 345, 346, 347, 348, 349, 350, 351, 354, 355, 360, 361, 362, 363, 364, 365, 366, 367, 368, 369, 370, 371, 372, 373, 374, 375, 376, 377, 378, 379, 380, 381, 384, 385, 386, 387, 388, 389, 392, 393, 394, 395, 396, 397, 400, 401, 402, 403, 404, 405, 408, 409, 410, 411, 412, 413, 414, 415, 416, 417, 418, 419, 420, 421, 422, 423, 426, 427, 428, 429, 432, 433, 434, 435, 438, 439, 440, 441, 442, 443, 444, 445, 446, 447, 448, 449, 450, 451, 452, 453, 454, 455, 456, 457, 462, 463, 468, 469, 470, 471, 476, 477, 478, 479, 480, 481, 482, 483, 492, 493, 494, 495, 496, 497, 498, 499, 500, 502, 504, 506, 508, 509, 510, 511, 512, 514, 516, 522, 523, 524, 525, 526, 527, 528, 529, 530, 531, 532, 533, 536, 537, 538, 539, 540, 541, 542, 543};
#endif
