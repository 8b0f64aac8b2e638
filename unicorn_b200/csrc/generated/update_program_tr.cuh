// Generated by unicorn_b200/mech/codegen.py: the in-place species-update program
// (src/lib/solvesp.f:85-2806) for a tile whose RC block is held on chip.
// RC rows: 256 in tensor memory (row i in columns 2i, 2i+1: low and high
// word), 281 in shared memory. Requires RCS(i) (shared-memory row i of the
// cell), TM_LD(bank, q, col) (load the double at column col into slot q of a
// register bank), TM_WAIT(bank) (wait for the loads of that bank), RCT(bank, q),
// UC_TR_PF(slot, k) (fetch Y0, FACE_SUM and FACE_NBR of species k into register slot 0
// or 1; read as Y0S, FSS, FNS), UC_TR_SYNC() (after every species: a barrier or nothing)
// and the accessors of the in-place program (YO, YN, YOS, SOUR, WM, UC_UPDATE_TAIL;
// scalars rho, dt, sor1, sor2, rsd). The production, extra and loss statements of a
// species are interleaved; each sum keeps the reference's order.
// 74 segments and 886 tensor-memory loads per cell and pass.
#pragma once
#define UC_TR_NT 256
#define UC_TR_NS 281
#define UC_TR_SEG 12
#define UC_TR_SHADOW_SAVE() do { YOS(0) = YO(2); YOS(1) = YO(4); YOS(2) = YO(6); YOS(3) = YO(13); YOS(4) = YO(16); YOS(5) = YO(14); YOS(6) = YO(8); YOS(7) = YO(22); } while (0)
#define UC_UPDATE_PROGRAM_TR() do { \
    double prod = 0.0, extra, loss, rhs1, rhs2, ppp, fnew; \
    TM_LD(0, 0, 6); \
    TM_LD(0, 1, 4); \
    TM_LD(0, 2, 10); \
    TM_LD(0, 3, 8); \
    TM_LD(0, 4, 16); \
    TM_LD(0, 5, 18); \
    TM_LD(0, 6, 44); \
    TM_LD(0, 7, 46); \
    TM_LD(0, 8, 68); \
    TM_LD(0, 9, 70); \
    TM_LD(0, 10, 100); \
    TM_LD(0, 11, 102); \
    TM_WAIT(0); \
    TM_LD(1, 0, 128); \
    TM_LD(1, 1, 130); \
    TM_LD(1, 2, 148); \
    TM_LD(1, 3, 150); \
    TM_LD(1, 4, 168); \
    TM_LD(1, 5, 170); \
    TM_LD(1, 6, 172); \
    TM_LD(1, 7, 174); \
    TM_LD(1, 8, 200); \
    TM_LD(1, 9, 202); \
    TM_LD(1, 10, 228); \
    TM_LD(1, 11, 230); \
    UC_TR_PF(0, 0); \
    UC_TR_PF(1, 1); \
    prod = ((YO(4) * YO(2)) * RCT(0, 0)); \
    extra = (1.0 * ((YO(46) * YO(2)) * RCS(251))); \
    loss = (YO(3) * RCT(0, 1)); \
    prod = prod + ((YO(5) * YO(2)) * RCT(0, 2)); \
    extra = extra + (1.0 * ((YO(46) * YO(2)) * RCS(252))); \
    loss = loss + (YO(4) * RCT(0, 3)); \
    prod = prod + ((YO(2) * YO(2)) * RCT(0, 4)); \
    extra = extra + (1.0 * ((YO(46) * YO(2)) * RCS(253))); \
    loss = loss + RCT(0, 5); \
    prod = prod + ((YO(6) * YO(2)) * RCT(0, 6)); \
    loss = loss + (YO(1) * RCT(0, 7)); \
    prod = prod + ((YO(7) * YO(2)) * RCT(0, 8)); \
    loss = loss + (YO(6) * RCT(0, 9)); \
    prod = prod + ((YO(10) * YO(2)) * RCT(0, 10)); \
    loss = loss + (YO(8) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 240); \
    TM_LD(0, 1, 242); \
    TM_LD(0, 2, 244); \
    TM_LD(0, 3, 246); \
    TM_LD(0, 4, 264); \
    TM_LD(0, 5, 266); \
    TM_LD(0, 6, 288); \
    TM_LD(0, 7, 290); \
    TM_LD(0, 8, 312); \
    TM_LD(0, 9, 314); \
    TM_LD(0, 10, 332); \
    TM_LD(0, 11, 334); \
    prod = prod + ((YO(11) * YO(2)) * RCT(1, 0)); \
    loss = loss + (YO(10) * RCT(1, 1)); \
    prod = prod + ((YO(12) * YO(2)) * RCT(1, 2)); \
    loss = loss + (YO(13) * RCT(1, 3)); \
    prod = prod + ((YO(13) * YO(2)) * RCT(1, 4)); \
    loss = loss + (YO(14) * RCT(1, 5)); \
    prod = prod + ((YO(13) * YO(2)) * RCT(1, 6)); \
    loss = loss + (YO(15) * RCT(1, 7)); \
    prod = prod + ((YO(13) * YO(13)) * RCT(1, 8)); \
    loss = loss + (YO(16) * RCT(1, 9)); \
    prod = prod + ((YO(14) * YO(2)) * RCT(1, 10)); \
    loss = loss + (YO(20) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 364); \
    TM_LD(1, 1, 366); \
    TM_LD(1, 2, 368); \
    TM_LD(1, 3, 370); \
    TM_LD(1, 4, 2); \
    TM_LD(1, 5, 0); \
    TM_LD(1, 6, 24); \
    TM_LD(1, 7, 26); \
    TM_LD(1, 8, 38); \
    TM_LD(1, 9, 36); \
    TM_LD(1, 10, 44); \
    TM_LD(1, 11, 46); \
    prod = prod + ((YO(14) * YO(3)) * RCT(0, 0)); \
    loss = loss + (YO(8) * RCT(0, 1)); \
    prod = prod + ((YO(14) * YO(1)) * RCT(0, 2)); \
    loss = loss + (YO(9) * RCT(0, 3)); \
    prod = prod + ((YO(17) * YO(2)) * RCT(0, 4)); \
    loss = loss + (YO(11) * RCT(0, 5)); \
    prod = prod + ((YO(19) * YO(2)) * RCT(0, 6)); \
    loss = loss + (YO(18) * RCT(0, 7)); \
    prod = prod + ((YO(18) * YO(2)) * RCT(0, 8)); \
    loss = loss + (YO(16) * RCT(0, 9)); \
    prod = prod + ((YO(16) * YO(2)) * RCT(0, 10)); \
    loss = loss + (YO(22) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 52); \
    TM_LD(0, 1, 54); \
    TM_LD(0, 2, 56); \
    TM_LD(0, 3, 58); \
    TM_LD(0, 4, 64); \
    TM_LD(0, 5, 66); \
    TM_LD(0, 6, 94); \
    TM_LD(0, 7, 92); \
    TM_LD(0, 8, 118); \
    TM_LD(0, 9, 116); \
    TM_LD(0, 10, 142); \
    TM_LD(0, 11, 140); \
    prod = prod + (YO(16) * RCT(1, 0)); \
    loss = loss + (YO(21) * RCT(1, 1)); \
    prod = prod + ((YO(22) * YO(2)) * RCT(1, 2)); \
    loss = loss + (YO(21) * RCT(1, 3)); \
    prod = prod + ((YO(28) * YO(2)) * RCS(50)); \
    loss = loss + (YO(11) * RCS(51)); \
    prod = prod + ((YO(29) * YO(2)) * RCS(64)); \
    loss = loss + (YO(28) * RCS(65)); \
    prod = prod + ((YO(29) * YO(2)) * RCS(66)); \
    loss = loss + (YO(17) * RCS(67)); \
    prod = prod + ((YO(23) * YO(2)) * RCS(76)); \
    loss = loss + (YO(25) * RCS(77)); \
    prod = prod + ((YO(31) * YO(2)) * RCS(98)); \
    loss = loss + (YO(34) * RCS(99)); \
    prod = prod + ((YO(31) * YO(2)) * RCS(100)); \
    loss = loss + (YO(23) * RCS(101)); \
    prod = prod + ((YO(30) * YO(2)) * RCS(118)); \
    loss = loss + (YO(33) * RCS(119)); \
    prod = prod + ((YO(30) * YO(2)) * RCS(120)); \
    loss = loss + (YO(32) * RCS(121)); \
    prod = prod + ((YO(30) * YO(2)) * RCS(122)); \
    loss = loss + (YO(35) * RCS(123)); \
    prod = prod + ((YO(38) * YO(2)) * RCS(178)); \
    loss = loss + (YO(36) * RCS(179)); \
    prod = prod + ((YO(39) * YO(2)) * RCS(198)); \
    loss = loss + (YO(38) * RCS(199)); \
    prod = prod + ((YO(40) * YO(2)) * RCS(212)); \
    loss = loss + (YO(41) * RCS(213)); \
    prod = prod + ((YO(40) * YO(2)) * RCS(214)); \
    loss = loss + (YO(42) * RCS(215)); \
    prod = prod + ((YO(43) * YO(2)) * RCS(236)); \
    loss = loss + ((YO(21) * YO(22)) * RCS(237)); \
    prod = prod + ((YO(46) * YO(2)) * RCS(254)); \
    loss = loss + ((YO(48) * YO(18)) * RCS(255)); \
    prod = prod + ((YO(48) * YO(2)) * RCS(263)); \
    loss = loss + ((YO(39) * YO(22)) * RCS(264)); \
    prod = prod + ((YO(48) * YO(2)) * RCS(269)); \
    loss = loss + ((YO(16) * YO(38)) * RCS(270)); \
    prod = prod + ((YO(48) * YO(2)) * RCS(271)); \
    loss = loss + ((YO(43) * YO(13)) * RCS(272)); \
    prod = prod + ((YO(47) * YO(2)) * RCS(277)); \
    loss = loss + ((YO(22) * YO(16)) * RCS(278)); \
    prod = prod + (SOUR(0) * YO(21)); \
    rhs1 = rho * Y0S(0) + dt * WM(0) * (prod + extra); \
    rhs2 = -(dt * WM(0) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(0) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(0) - fnew); \
    UC_UPDATE_TAIL(0); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 2); \
    prod = ((YO(4) * YO(3)) * RCT(1, 4)); \
    extra = 0.0; \
    loss = (YO(2) * RCT(1, 5)); \
    prod = prod + ((YO(3) * YO(3)) * RCT(1, 6)); \
    loss = loss + RCT(1, 7); \
    prod = prod + (YO(6) * RCT(1, 8)); \
    loss = loss + (YO(2) * RCT(1, 9)); \
    prod = prod + ((YO(6) * YO(2)) * RCT(1, 10)); \
    loss = loss + (YN(0) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 162); \
    TM_LD(1, 1, 160); \
    TM_LD(1, 2, 194); \
    TM_LD(1, 3, 192); \
    TM_LD(1, 4, 198); \
    TM_LD(1, 5, 196); \
    TM_LD(1, 6, 246); \
    TM_LD(1, 7, 244); \
    TM_LD(1, 8, 254); \
    TM_LD(1, 9, 252); \
    TM_LD(1, 10, 282); \
    TM_LD(1, 11, 280); \
    prod = prod + ((YO(6) * YO(3)) * RCT(0, 0)); \
    loss = loss + (YO(4) * RCT(0, 1)); \
    prod = prod + ((YO(6) * YO(4)) * RCT(0, 2)); \
    loss = loss + (YO(5) * RCT(0, 3)); \
    prod = prod + ((YO(6) * YO(6)) * RCT(0, 4)); \
    loss = loss + (YO(7) * RCT(0, 5)); \
    prod = prod + ((YO(9) * YO(3)) * RCT(0, 6)); \
    loss = loss + (YO(8) * RCT(0, 7)); \
    prod = prod + ((YO(8) * YO(6)) * RCT(0, 8)); \
    loss = loss + (YO(10) * RCT(0, 9)); \
    prod = prod + ((YO(10) * YO(6)) * RCT(0, 10)); \
    loss = loss + (YO(11) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 326); \
    TM_LD(0, 1, 324); \
    TM_LD(0, 2, 354); \
    TM_LD(0, 3, 352); \
    TM_LD(0, 4, 378); \
    TM_LD(0, 5, 376); \
    TM_LD(0, 6, 382); \
    TM_LD(0, 7, 380); \
    TM_LD(0, 8, 2); \
    TM_LD(0, 9, 0); \
    TM_LD(0, 10, 4); \
    TM_LD(0, 11, 6); \
    prod = prod + ((YO(13) * YO(6)) * RCT(1, 0)); \
    loss = loss + (YO(12) * RCT(1, 1)); \
    prod = prod + ((YO(11) * YO(4)) * RCT(1, 2)); \
    loss = loss + (YO(13) * RCT(1, 3)); \
    prod = prod + ((YO(17) * YO(3)) * RCT(1, 4)); \
    loss = loss + (YO(13) * RCT(1, 5)); \
    prod = prod + (((YO(8) * YO(4)) * YO(2)) * RCS(1)); \
    loss = loss + (YO(15) * RCS(0)); \
    prod = prod + (YN(0) * (YO(9) * RCT(1, 6))); \
    loss = loss + (YO(14) * RCT(1, 7)); \
    prod = prod + (((YO(8) * YO(4)) * YO(2)) * RCS(5)); \
    loss = loss + (YO(14) * RCS(4)); \
    prod = prod + ((YO(10) * YO(3)) * RCT(1, 8)); \
    loss = loss + (YO(20) * RCT(1, 9)); \
    prod = prod + ((YO(11) * YO(6)) * RCT(1, 10)); \
    loss = loss + (YO(17) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 8); \
    TM_LD(1, 1, 10); \
    TM_LD(1, 2, 18); \
    TM_LD(1, 3, 16); \
    TM_LD(1, 4, 22); \
    TM_LD(1, 5, 20); \
    TM_LD(1, 6, 30); \
    TM_LD(1, 7, 28); \
    TM_LD(1, 8, 38); \
    TM_LD(1, 9, 36); \
    TM_LD(1, 10, 42); \
    TM_LD(1, 11, 40); \
    prod = prod + ((YO(16) * YO(6)) * RCT(0, 0)); \
    loss = loss + (YO(18) * RCT(0, 1)); \
    prod = prod + ((YO(22) * YO(6)) * RCT(0, 2)); \
    loss = loss + (YO(16) * RCT(0, 3)); \
    prod = prod + ((YO(11) * YO(10)) * RCT(0, 4)); \
    loss = loss + (YO(22) * RCT(0, 5)); \
    prod = prod + ((YO(23) * YO(3)) * RCT(0, 6)); \
    loss = loss + (YO(22) * RCT(0, 7)); \
    prod = prod + ((YO(21) * YO(6)) * RCS(11)); \
    loss = loss + (YO(22) * RCS(10)); \
    prod = prod + ((YO(11) * YO(8)) * RCS(17)); \
    loss = loss + (YO(21) * RCS(16)); \
    prod = prod + (((YO(8) * YO(8)) * YO(4)) * RCS(37)); \
    loss = loss + (YO(26) * RCS(36)); \
    prod = prod + (((YO(9) * YO(8)) * YO(2)) * RCS(39)); \
    loss = loss + (YO(26) * RCS(38)); \
    prod = prod + ((YO(26) * YO(3)) * RCS(45)); \
    loss = loss + (YO(27) * RCS(44)); \
    prod = prod + ((YO(20) * YO(9)) * RCS(47)); \
    loss = loss + (YO(27) * RCS(46)); \
    prod = prod + ((YO(10) * YO(8)) * RCS(49)); \
    loss = loss + (YO(27) * RCS(48)); \
    prod = prod + ((YO(11) * YO(6)) * RCS(57)); \
    loss = loss + (YO(28) * RCS(56)); \
    prod = prod + ((YO(28) * YO(6)) * RCS(73)); \
    loss = loss + (YO(29) * RCS(72)); \
    prod = prod + (((YO(11) * YO(8)) * YO(4)) * RCS(83)); \
    loss = loss + (YO(23) * RCS(82)); \
    prod = prod + ((YO(23) * YO(6)) * RCS(88)); \
    loss = loss + (YO(31) * RCS(89)); \
    prod = prod + ((YO(34) * YO(6)) * RCS(111)); \
    loss = loss + (YO(31) * RCS(110)); \
    prod = prod + ((YO(31) * YO(6)) * RCS(145)); \
    loss = loss + (YO(35) * RCS(144)); \
    prod = prod + ((YO(31) * YO(6)) * RCS(155)); \
    loss = loss + (YO(32) * RCS(154)); \
    prod = prod + ((YO(37) * YO(6)) * RCS(172)); \
    loss = loss + (YO(36) * RCS(173)); \
    prod = prod + ((YO(25) * YO(10)) * RCS(177)); \
    loss = loss + (YO(37) * RCS(176)); \
    prod = prod + ((YO(36) * YO(6)) * RCS(181)); \
    loss = loss + (YO(38) * RCS(180)); \
    prod = prod + (((YO(13) * YO(10)) * YO(8)) * RCS(191)); \
    loss = loss + (YO(36) * RCS(190)); \
    prod = prod + ((YO(38) * YO(6)) * RCS(200)); \
    loss = loss + (YO(39) * RCS(201)); \
    prod = prod + ((YO(41) * YO(6)) * RCS(209)); \
    loss = loss + (YO(40) * RCS(208)); \
    prod = prod + ((YO(42) * YO(6)) * RCS(211)); \
    loss = loss + (YO(40) * RCS(210)); \
    prod = prod + ((YO(39) * YO(6)) * RCS(229)); \
    loss = loss + (YO(41) * RCS(228)); \
    prod = prod + ((YO(39) * YO(6)) * RCS(231)); \
    loss = loss + (YO(42) * RCS(230)); \
    prod = prod + (((YO(21) * YO(38)) * YO(6)) * RCS(243)); \
    loss = loss + (YO(45) * RCS(242)); \
    prod = prod + (((YO(22) * YO(36)) * YO(6)) * RCS(245)); \
    loss = loss + (YO(45) * RCS(244)); \
    loss = loss + (0.5 * SOUR(2)); \
    rhs1 = rho * Y0S(1) + dt * WM(1) * (prod + extra); \
    rhs2 = -(dt * WM(1) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(1) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(1) - fnew); \
    UC_UPDATE_TAIL(1); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 3); \
    prod = ((YO(4) * YO(3)) * RCT(0, 8)); \
    extra = 0.0; \
    loss = (YN(1) * RCT(0, 9)); \
    prod = prod + (YN(0) * (YO(3) * RCT(0, 10))); \
    loss = loss + (YO(4) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 46); \
    TM_LD(0, 1, 44); \
    TM_LD(0, 2, 50); \
    TM_LD(0, 3, 48); \
    TM_LD(0, 4, 70); \
    TM_LD(0, 5, 68); \
    TM_LD(0, 6, 74); \
    TM_LD(0, 7, 72); \
    TM_LD(0, 8, 84); \
    TM_LD(0, 9, 86); \
    TM_LD(0, 10, 96); \
    TM_LD(0, 11, 98); \
    prod = prod + (YN(0) * (YO(4) * RCT(1, 0))); \
    loss = loss + (YO(5) * RCT(1, 1)); \
    prod = prod + (YN(0) * RCT(1, 2)); \
    loss = loss + (YO(2) * RCT(1, 3)); \
    prod = prod + (YN(0) * RCT(1, 2)); \
    loss = loss + (YO(2) * RCT(1, 3)); \
    prod = prod + (YO(5) * RCT(1, 4)); \
    loss = loss + (YO(4) * RCT(1, 5)); \
    prod = prod + (YO(4) * RCT(1, 6)); \
    loss = loss + (YO(3) * RCT(1, 7)); \
    prod = prod + (YO(6) * RCT(1, 8)); \
    loss = loss + (YN(1) * RCT(1, 9)); \
    prod = prod + ((YO(4) * YO(4)) * RCT(1, 10)); \
    loss = loss + (YO(6) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 102); \
    TM_LD(1, 1, 100); \
    TM_LD(1, 2, 108); \
    TM_LD(1, 3, 110); \
    TM_LD(1, 4, 126); \
    TM_LD(1, 5, 124); \
    TM_LD(1, 6, 130); \
    TM_LD(1, 7, 128); \
    TM_LD(1, 8, 150); \
    TM_LD(1, 9, 148); \
    TM_LD(1, 10, 170); \
    TM_LD(1, 11, 168); \
    prod = prod + (YN(1) * (YN(0) * RCT(0, 0))); \
    loss = loss + (YO(6) * RCT(0, 1)); \
    prod = prod + ((YO(5) * YO(3)) * RCT(0, 2)); \
    loss = loss + (YO(6) * RCT(0, 3)); \
    prod = prod + (YN(0) * (YO(6) * RCT(0, 4))); \
    loss = loss + (YO(7) * RCT(0, 5)); \
    prod = prod + ((YO(5) * YO(4)) * RCT(0, 6)); \
    loss = loss + (YO(7) * RCT(0, 7)); \
    prod = prod + ((YO(8) * YO(4)) * RCT(0, 8)); \
    loss = loss + (YO(9) * RCT(0, 9)); \
    prod = prod + (YO(10) * RCT(0, 10)); \
    loss = loss + (YO(8) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 174); \
    TM_LD(0, 1, 172); \
    TM_LD(0, 2, 180); \
    TM_LD(0, 3, 182); \
    TM_LD(0, 4, 184); \
    TM_LD(0, 5, 186); \
    TM_LD(0, 6, 204); \
    TM_LD(0, 7, 206); \
    TM_LD(0, 8, 210); \
    TM_LD(0, 9, 208); \
    TM_LD(0, 10, 216); \
    TM_LD(0, 11, 218); \
    prod = prod + (YN(0) * (YO(8) * RCT(1, 0))); \
    loss = loss + (YO(10) * RCT(1, 1)); \
    prod = prod + ((YO(10) * YO(3)) * RCT(1, 2)); \
    loss = loss + (YO(9) * RCT(1, 3)); \
    prod = prod + (YO(11) * RCT(1, 4)); \
    loss = loss + (YO(10) * RCT(1, 5)); \
    prod = prod + (YN(0) * (YO(10) * RCT(1, 6))); \
    loss = loss + (YO(11) * RCT(1, 7)); \
    prod = prod + (YN(0) * (YO(13) * RCT(1, 8))); \
    loss = loss + (YO(12) * RCT(1, 9)); \
    prod = prod + (YN(0) * (YO(14) * RCT(1, 10))); \
    loss = loss + (YO(13) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 230); \
    TM_LD(1, 1, 228); \
    TM_LD(1, 2, 232); \
    TM_LD(1, 3, 234); \
    TM_LD(1, 4, 248); \
    TM_LD(1, 5, 250); \
    TM_LD(1, 6, 256); \
    TM_LD(1, 7, 258); \
    TM_LD(1, 8, 266); \
    TM_LD(1, 9, 264); \
    TM_LD(1, 10, 270); \
    TM_LD(1, 11, 268); \
    prod = prod + (YN(0) * (YO(15) * RCT(0, 0))); \
    loss = loss + (YO(13) * RCT(0, 1)); \
    prod = prod + ((YO(13) * YO(3)) * RCT(0, 2)); \
    loss = loss + (YO(11) * RCT(0, 3)); \
    prod = prod + ((YO(13) * YO(14)) * RCT(0, 4)); \
    loss = loss + (YO(16) * RCT(0, 5)); \
    prod = prod + ((YO(13) * YO(13)) * RCT(0, 6)); \
    loss = loss + (YO(18) * RCT(0, 7)); \
    prod = prod + (YO(12) * RCT(0, 8)); \
    loss = loss + (YO(13) * RCT(0, 9)); \
    prod = prod + ((YO(15) * YO(4)) * RCT(0, 10)); \
    loss = loss + (YO(11) * RCT(0, 11)); \
    prod = prod + (YN(1) * (YO(15) * RCS(0))); \
    loss = loss + ((YO(8) * YO(4)) * RCS(1)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 284); \
    TM_LD(0, 1, 286); \
    TM_LD(0, 2, 290); \
    TM_LD(0, 3, 288); \
    TM_LD(0, 4, 304); \
    TM_LD(0, 5, 306); \
    TM_LD(0, 6, 314); \
    TM_LD(0, 7, 312); \
    TM_LD(0, 8, 328); \
    TM_LD(0, 9, 330); \
    TM_LD(0, 10, 334); \
    TM_LD(0, 11, 332); \
    prod = prod + (YN(0) * (YO(20) * RCT(1, 0))); \
    loss = loss + (YO(14) * RCT(1, 1)); \
    prod = prod + ((YO(14) * YO(4)) * RCT(1, 2)); \
    loss = loss + (YO(11) * RCT(1, 3)); \
    prod = prod + ((YO(14) * YO(3)) * RCS(2)); \
    loss = loss + ((YO(8) * YO(2)) * RCS(3)); \
    prod = prod + ((YO(14) * YO(3)) * RCS(2)); \
    loss = loss + ((YO(8) * YO(2)) * RCS(3)); \
    prod = prod + (YN(1) * (YO(14) * RCS(4))); \
    loss = loss + ((YO(8) * YO(4)) * RCS(5)); \
    prod = prod + ((YO(14) * YO(14)) * RCS(6)); \
    loss = loss + ((YO(21) * YO(2)) * RCS(7)); \
    prod = prod + ((YO(14) * YO(14)) * RCS(6)); \
    loss = loss + ((YO(21) * YO(2)) * RCS(7)); \
    prod = prod + ((YO(20) * YO(3)) * RCT(1, 4)); \
    loss = loss + (YO(8) * RCT(1, 5)); \
    prod = prod + ((YO(20) * YO(5)) * RCT(1, 6)); \
    loss = loss + (YO(11) * RCT(1, 7)); \
    prod = prod + (YN(0) * (YO(11) * RCT(1, 8))); \
    loss = loss + (YO(17) * RCT(1, 9)); \
    prod = prod + ((YO(15) * YO(5)) * RCT(1, 10)); \
    loss = loss + (YO(17) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 344); \
    TM_LD(1, 1, 346); \
    TM_LD(1, 2, 360); \
    TM_LD(1, 3, 362); \
    TM_LD(1, 4, 370); \
    TM_LD(1, 5, 368); \
    TM_LD(1, 6, 372); \
    TM_LD(1, 7, 374); \
    TM_LD(1, 8, 384); \
    TM_LD(1, 9, 386); \
    TM_LD(1, 10, 396); \
    TM_LD(1, 11, 398); \
    prod = prod + (YO(17) * RCT(0, 0)); \
    loss = loss + (YO(11) * RCT(0, 1)); \
    prod = prod + (YN(0) * (YO(18) * RCT(0, 2))); \
    loss = loss + (YO(19) * RCT(0, 3)); \
    prod = prod + (YO(19) * RCT(0, 4)); \
    loss = loss + (YO(18) * RCT(0, 5)); \
    prod = prod + (YN(0) * (YO(16) * RCT(0, 6))); \
    loss = loss + (YO(18) * RCT(0, 7)); \
    prod = prod + (YO(18) * RCT(0, 8)); \
    loss = loss + (YO(16) * RCT(0, 9)); \
    prod = prod + (YN(0) * (YO(22) * RCT(0, 10))); \
    loss = loss + (YO(16) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 424); \
    TM_LD(0, 1, 426); \
    TM_LD(0, 2, 432); \
    TM_LD(0, 3, 434); \
    TM_LD(0, 4, 438); \
    TM_LD(0, 5, 436); \
    TM_LD(0, 6, 442); \
    TM_LD(0, 7, 440); \
    TM_LD(0, 8, 450); \
    TM_LD(0, 9, 448); \
    TM_LD(0, 10, 466); \
    TM_LD(0, 11, 464); \
    prod = prod + ((YO(16) * YO(3)) * RCT(1, 0)); \
    loss = loss + (YO(23) * RCT(1, 1)); \
    prod = prod + (YO(16) * RCT(1, 2)); \
    loss = loss + (YO(22) * RCT(1, 3)); \
    prod = prod + (YN(0) * (YO(21) * RCT(1, 4))); \
    loss = loss + (YO(22) * RCT(1, 5)); \
    prod = prod + (YO(22) * RCT(1, 6)); \
    loss = loss + (YO(21) * RCT(1, 7)); \
    prod = prod + ((YO(21) * YO(3)) * RCS(12)); \
    loss = loss + (YO(26) * RCS(13)); \
    prod = prod + ((YO(21) * YO(4)) * RCS(18)); \
    loss = loss + (YO(25) * RCS(19)); \
    prod = prod + ((YO(13) * YO(8)) * RCS(23)); \
    loss = loss + (YO(25) * RCS(22)); \
    prod = prod + ((YO(15) * YO(8)) * RCS(31)); \
    loss = loss + (YO(26) * RCS(30)); \
    prod = prod + ((YO(26) * YO(4)) * RCS(32)); \
    loss = loss + ((YO(10) * YO(8)) * RCS(33)); \
    prod = prod + ((YO(26) * YO(3)) * RCS(34)); \
    loss = loss + ((YO(8) * YO(8)) * RCS(35)); \
    prod = prod + (YN(1) * (YO(26) * RCS(38))); \
    loss = loss + ((YO(9) * YO(8)) * RCS(39)); \
    prod = prod + ((YO(27) * YO(4)) * RCS(40)); \
    loss = loss + (YO(26) * RCS(41)); \
    prod = prod + (YN(0) * (YO(11) * RCS(51))); \
    loss = loss + (YO(28) * RCS(50)); \
    prod = prod + ((YO(13) * YO(4)) * RCS(53)); \
    loss = loss + (YO(28) * RCS(52)); \
    prod = prod + (YO(28) * RCT(1, 8)); \
    loss = loss + (YO(11) * RCT(1, 9)); \
    prod = prod + (YN(0) * (YO(28) * RCS(65))); \
    loss = loss + (YO(29) * RCS(64)); \
    prod = prod + (YN(0) * (YO(17) * RCS(67))); \
    loss = loss + (YO(29) * RCS(66)); \
    prod = prod + (YO(23) * RCT(1, 10)); \
    loss = loss + (YO(25) * RCT(1, 11)); \
    prod = prod + ((YO(13) * YO(10)) * RCS(75)); \
    loss = loss + (YO(23) * RCS(74)); \
    prod = prod + (YN(0) * (YO(25) * RCS(77))); \
    loss = loss + (YO(23) * RCS(76)); \
    prod = prod + ((YO(23) * YO(13)) * RCS(84)); \
    loss = loss + ((YO(18) * YO(8)) * RCS(85)); \
    prod = prod + (YN(0) * (YO(34) * RCS(99))); \
    loss = loss + (YO(31) * RCS(98)); \
    prod = prod + (YN(0) * (YO(23) * RCS(101))); \
    loss = loss + (YO(31) * RCS(100)); \
    prod = prod + (YN(0) * (YO(33) * RCS(119))); \
    loss = loss + (YO(30) * RCS(118)); \
    prod = prod + (YN(0) * (YO(32) * RCS(121))); \
    loss = loss + (YO(30) * RCS(120)); \
    prod = prod + (YN(0) * (YO(35) * RCS(123))); \
    loss = loss + (YO(30) * RCS(122)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 474); \
    TM_LD(1, 1, 472); \
    TM_LD(1, 2, 0); \
    TM_LD(1, 3, 2); \
    TM_LD(1, 4, 6); \
    TM_LD(1, 5, 4); \
    TM_LD(1, 6, 14); \
    TM_LD(1, 7, 12); \
    TM_LD(1, 8, 26); \
    TM_LD(1, 9, 24); \
    TM_LD(1, 10, 30); \
    TM_LD(1, 11, 28); \
    prod = prod + (YO(35) * RCT(0, 0)); \
    loss = loss + (YO(31) * RCT(0, 1)); \
    prod = prod + ((YO(13) * YO(28)) * RCS(149)); \
    loss = loss + (YO(35) * RCS(148)); \
    prod = prod + ((YO(16) * YO(5)) * RCS(151)); \
    loss = loss + (YO(35) * RCS(150)); \
    prod = prod + ((YO(16) * YO(5)) * RCS(159)); \
    loss = loss + (YO(32) * RCS(158)); \
    prod = prod + ((YO(13) * YO(28)) * RCS(161)); \
    loss = loss + (YO(32) * RCS(160)); \
    prod = prod + (YO(32) * RCT(0, 2)); \
    loss = loss + (YO(31) * RCT(0, 3)); \
    prod = prod + ((YO(13) * YO(21)) * RCS(168)); \
    loss = loss + (YO(36) * RCS(169)); \
    prod = prod + (YO(36) * RCT(0, 4)); \
    loss = loss + (YO(37) * RCT(0, 5)); \
    prod = prod + (YO(38) * RCT(0, 6)); \
    loss = loss + (YO(36) * RCT(0, 7)); \
    prod = prod + (YN(0) * (YO(36) * RCS(179))); \
    loss = loss + (YO(38) * RCS(178)); \
    prod = prod + ((YO(39) * YO(3)) * RCS(196)); \
    loss = loss + ((YO(25) * YO(13)) * RCS(197)); \
    prod = prod + (YN(0) * (YO(38) * RCS(199))); \
    loss = loss + (YO(39) * RCS(198)); \
    prod = prod + (YO(39) * RCT(0, 8)); \
    loss = loss + (YO(38) * RCT(0, 9)); \
    prod = prod + ((YO(16) * YO(13)) * RCS(205)); \
    loss = loss + (YO(39) * RCS(204)); \
    prod = prod + ((YO(13) * YO(22)) * RCS(206)); \
    loss = loss + (YO(38) * RCS(207)); \
    prod = prod + (YN(0) * (YO(41) * RCS(213))); \
    loss = loss + (YO(40) * RCS(212)); \
    prod = prod + (YN(0) * (YO(42) * RCS(215))); \
    loss = loss + (YO(40) * RCS(214)); \
    prod = prod + (YO(41) * RCT(0, 10)); \
    loss = loss + (YO(39) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 34); \
    TM_LD(0, 1, 32); \
    TM_LD(0, 2, 48); \
    TM_LD(0, 3, 50); \
    TM_LD(0, 4, 54); \
    TM_LD(0, 5, 52); \
    TM_LD(0, 6, 82); \
    TM_LD(0, 7, 80); \
    TM_LD(0, 8, 92); \
    TM_LD(0, 9, 94); \
    TM_LD(0, 10, 106); \
    TM_LD(0, 11, 104); \
    prod = prod + (YO(42) * RCT(1, 0)); \
    loss = loss + (YO(39) * RCT(1, 1)); \
    prod = prod + (YO(43) * RCS(232)); \
    loss = loss + ((YO(21) * YO(22)) * RCS(233)); \
    prod = prod + ((YO(22) * YO(16)) * RCS(235)); \
    loss = loss + (YO(43) * RCS(234)); \
    prod = prod + (YN(0) * ((YO(21) * YO(22)) * RCS(237))); \
    loss = loss + (YO(43) * RCS(236)); \
    prod = prod + ((YO(43) * YO(4)) * RCS(238)); \
    loss = loss + ((YO(44) * YO(38)) * RCS(239)); \
    prod = prod + 0.0; \
    loss = loss + (YO(46) * RCS(251)); \
    prod = prod + 0.0; \
    loss = loss + (YO(46) * RCS(252)); \
    prod = prod + 0.0; \
    loss = loss + (YO(46) * RCS(253)); \
    prod = prod + (YN(0) * ((YO(48) * YO(18)) * RCS(255))); \
    loss = loss + (YO(46) * RCS(254)); \
    prod = prod + (YN(0) * ((YO(39) * YO(22)) * RCS(264))); \
    loss = loss + (YO(48) * RCS(263)); \
    prod = prod + (((YO(16) * YO(16)) * YO(13)) * RCS(266)); \
    loss = loss + (YO(48) * RCS(265)); \
    prod = prod + ((YO(39) * YO(18)) * RCS(268)); \
    loss = loss + (YO(48) * RCS(267)); \
    prod = prod + (YN(0) * ((YO(16) * YO(38)) * RCS(270))); \
    loss = loss + (YO(48) * RCS(269)); \
    prod = prod + (YN(0) * ((YO(43) * YO(13)) * RCS(272))); \
    loss = loss + (YO(48) * RCS(271)); \
    prod = prod + ((YO(16) * YO(18)) * RCS(274)); \
    loss = loss + (YO(47) * RCS(273)); \
    prod = prod + ((YO(39) * YO(13)) * RCS(276)); \
    loss = loss + (YO(47) * RCS(275)); \
    prod = prod + (YN(0) * ((YO(22) * YO(16)) * RCS(278))); \
    loss = loss + (YO(47) * RCS(277)); \
    prod = prod + ((YO(47) * YO(4)) * RCS(279)); \
    loss = loss + ((YO(5) * YO(43)) * RCS(280)); \
    prod = prod + (SOUR(3) * YO(4)); \
    rhs1 = rho * Y0S(0) + dt * WM(2) * (prod + extra); \
    rhs2 = -(dt * WM(2) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(2) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(2) - fnew); \
    UC_UPDATE_TAIL(2); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 4); \
    prod = (YN(2) * (YN(1) * RCT(1, 2))); \
    extra = 0.0; \
    loss = (YO(4) * RCT(1, 3)); \
    prod = prod + (YN(2) * (YO(4) * RCT(1, 4))); \
    loss = loss + (YN(0) * RCT(1, 5)); \
    prod = prod + ((YO(4) * YO(4)) * RCT(1, 6)); \
    loss = loss + (YO(5) * RCT(1, 7)); \
    prod = prod + (YN(1) * RCT(1, 8)); \
    loss = loss + (YO(3) * RCT(1, 9)); \
    prod = prod + (YN(1) * RCT(1, 8)); \
    loss = loss + (YO(3) * RCT(1, 9)); \
    prod = prod + (YO(4) * RCT(1, 10)); \
    loss = loss + (YN(2) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 110); \
    TM_LD(1, 1, 108); \
    TM_LD(1, 2, 134); \
    TM_LD(1, 3, 132); \
    TM_LD(1, 4, 158); \
    TM_LD(1, 5, 156); \
    TM_LD(1, 6, 182); \
    TM_LD(1, 7, 180); \
    TM_LD(1, 8, 196); \
    TM_LD(1, 9, 198); \
    TM_LD(1, 10, 242); \
    TM_LD(1, 11, 240); \
    prod = prod + (YO(6) * RCT(0, 0)); \
    loss = loss + (YO(4) * RCT(0, 1)); \
    prod = prod + (YN(2) * (YO(6) * RCT(0, 2))); \
    loss = loss + (YO(5) * RCT(0, 3)); \
    prod = prod + (YN(1) * (YO(4) * RCT(0, 4))); \
    loss = loss + (YO(6) * RCT(0, 5)); \
    prod = prod + ((YO(6) * YO(4)) * RCT(0, 6)); \
    loss = loss + (YO(7) * RCT(0, 7)); \
    prod = prod + (YN(1) * (YO(8) * RCT(0, 8))); \
    loss = loss + (YO(9) * RCT(0, 9)); \
    prod = prod + ((YO(8) * YO(4)) * RCT(0, 10)); \
    loss = loss + (YO(10) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 250); \
    TM_LD(0, 1, 248); \
    TM_LD(0, 2, 252); \
    TM_LD(0, 3, 254); \
    TM_LD(0, 4, 278); \
    TM_LD(0, 5, 276); \
    TM_LD(0, 6, 294); \
    TM_LD(0, 7, 292); \
    TM_LD(0, 8, 318); \
    TM_LD(0, 9, 316); \
    TM_LD(0, 10, 322); \
    TM_LD(0, 11, 320); \
    prod = prod + (YN(2) * (YO(9) * RCT(1, 0))); \
    loss = loss + (YO(10) * RCT(1, 1)); \
    prod = prod + ((YO(10) * YO(4)) * RCT(1, 2)); \
    loss = loss + (YO(11) * RCT(1, 3)); \
    prod = prod + ((YO(13) * YO(4)) * RCT(1, 4)); \
    loss = loss + (YO(12) * RCT(1, 5)); \
    prod = prod + (YN(2) * (YO(11) * RCT(1, 6))); \
    loss = loss + (YO(13) * RCT(1, 7)); \
    prod = prod + (YN(1) * (YO(13) * RCT(1, 8))); \
    loss = loss + (YO(17) * RCT(1, 9)); \
    prod = prod + (YN(2) * ((YO(8) * YOS(0)) * RCS(3))); \
    loss = loss + (YO(14) * RCS(2)); \
    prod = prod + (YN(0) * (YO(8) * RCT(1, 10))); \
    loss = loss + (YO(14) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 342); \
    TM_LD(1, 1, 340); \
    TM_LD(1, 2, 346); \
    TM_LD(1, 3, 344); \
    TM_LD(1, 4, 380); \
    TM_LD(1, 5, 382); \
    TM_LD(1, 6, 0); \
    TM_LD(1, 7, 2); \
    TM_LD(1, 8, 4); \
    TM_LD(1, 9, 6); \
    TM_LD(1, 10, 10); \
    TM_LD(1, 11, 8); \
    prod = prod + (YN(2) * (YO(8) * RCT(0, 0))); \
    loss = loss + (YO(20) * RCT(0, 1)); \
    prod = prod + (YN(1) * (YO(20) * RCT(0, 2))); \
    loss = loss + (YO(10) * RCT(0, 3)); \
    prod = prod + ((YO(4) * YO(11)) * RCT(0, 4)); \
    loss = loss + (YO(17) * RCT(0, 5)); \
    prod = prod + ((YO(18) * YO(4)) * RCT(0, 6)); \
    loss = loss + (YO(19) * RCT(0, 7)); \
    prod = prod + ((YO(16) * YO(4)) * RCT(0, 8)); \
    loss = loss + (YO(18) * RCT(0, 9)); \
    prod = prod + ((YO(13) * YO(11)) * RCT(0, 10)); \
    loss = loss + (YO(18) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 12); \
    TM_LD(0, 1, 14); \
    TM_LD(0, 2, 22); \
    TM_LD(0, 3, 20); \
    TM_LD(0, 4, 28); \
    TM_LD(0, 5, 30); \
    TM_LD(0, 6, 34); \
    TM_LD(0, 7, 32); \
    TM_LD(0, 8, 40); \
    TM_LD(0, 9, 42); \
    TM_LD(0, 10, 52); \
    TM_LD(0, 11, 54); \
    prod = prod + ((YO(13) * YO(10)) * RCT(1, 0)); \
    loss = loss + (YO(16) * RCT(1, 1)); \
    prod = prod + (YN(2) * (YO(23) * RCT(1, 2))); \
    loss = loss + (YO(16) * RCT(1, 3)); \
    prod = prod + (YN(1) * (YO(22) * RCT(1, 4))); \
    loss = loss + (YO(23) * RCT(1, 5)); \
    prod = prod + (YN(2) * (YO(26) * RCS(13))); \
    loss = loss + (YO(21) * RCS(12)); \
    prod = prod + ((YO(14) * YO(8)) * RCS(15)); \
    loss = loss + (YO(21) * RCS(14)); \
    prod = prod + ((YO(14) * YO(9)) * RCS(25)); \
    loss = loss + (YO(25) * RCS(24)); \
    prod = prod + ((YO(26) * YO(4)) * RCS(27)); \
    loss = loss + (YO(25) * RCS(26)); \
    prod = prod + (YN(2) * ((YO(8) * YO(8)) * RCS(35))); \
    loss = loss + (YO(26) * RCS(34)); \
    prod = prod + ((YO(8) * YO(20)) * RCS(43)); \
    loss = loss + (YO(27) * RCS(42)); \
    prod = prod + (YN(1) * (YO(27) * RCS(44))); \
    loss = loss + (YO(26) * RCS(45)); \
    prod = prod + ((YO(28) * YO(4)) * RCS(69)); \
    loss = loss + (YO(29) * RCS(68)); \
    prod = prod + ((YO(11) * YO(10)) * RCS(79)); \
    loss = loss + (YO(23) * RCS(78)); \
    prod = prod + ((YO(34) * YO(4)) * RCS(95)); \
    loss = loss + (YO(31) * RCS(94)); \
    prod = prod + ((YO(23) * YO(4)) * RCS(97)); \
    loss = loss + (YO(31) * RCS(96)); \
    prod = prod + ((YO(33) * YO(4)) * RCS(125)); \
    loss = loss + (YO(30) * RCS(124)); \
    prod = prod + ((YO(32) * YO(4)) * RCS(127)); \
    loss = loss + (YO(30) * RCS(126)); \
    prod = prod + ((YO(35) * YO(4)) * RCS(129)); \
    loss = loss + (YO(30) * RCS(128)); \
    prod = prod + ((YO(31) * YO(4)) * RCS(157)); \
    loss = loss + (YO(32) * RCS(156)); \
    prod = prod + ((YO(16) * YO(8)) * RCS(167)); \
    loss = loss + (YO(36) * RCS(166)); \
    prod = prod + ((YO(26) * YO(13)) * RCS(171)); \
    loss = loss + (YO(36) * RCS(170)); \
    prod = prod + ((YO(18) * YO(10)) * RCS(193)); \
    loss = loss + (YO(39) * RCS(192)); \
    prod = prod + (YN(2) * ((YO(25) * YO(13)) * RCS(197))); \
    loss = loss + (YO(39) * RCS(196)); \
    prod = prod + ((YO(41) * YO(4)) * RCS(217)); \
    loss = loss + (YO(40) * RCS(216)); \
    prod = prod + ((YO(42) * YO(4)) * RCS(219)); \
    loss = loss + (YO(40) * RCS(218)); \
    loss = loss + SOUR(4); \
    rhs1 = rho * Y0S(1) + dt * WM(3) * (prod + extra); \
    rhs2 = -(dt * WM(3) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(3) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(3) - fnew); \
    UC_UPDATE_TAIL(3); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 5); \
    prod = (YN(2) * (YN(1) * RCT(1, 6))); \
    extra = 0.0; \
    loss = (YN(3) * RCT(1, 7)); \
    prod = prod + (YN(3) * (YN(0) * RCT(1, 8))); \
    loss = loss + (YN(2) * RCT(1, 9)); \
    prod = prod + (YN(2) * (YO(5) * RCT(1, 10))); \
    loss = loss + (YN(0) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 58); \
    TM_LD(1, 1, 56); \
    TM_LD(1, 2, 62); \
    TM_LD(1, 3, 60); \
    TM_LD(1, 4, 72); \
    TM_LD(1, 5, 74); \
    TM_LD(1, 6, 78); \
    TM_LD(1, 7, 76); \
    TM_LD(1, 8, 80); \
    TM_LD(1, 9, 82); \
    TM_LD(1, 10, 86); \
    TM_LD(1, 11, 84); \
    prod = prod + (YN(3) * (YO(5) * RCT(0, 0))); \
    loss = loss + (YO(4) * RCT(0, 1)); \
    prod = prod + (YN(3) * (YO(5) * RCT(0, 0))); \
    loss = loss + (YO(4) * RCT(0, 1)); \
    prod = prod + (YO(5) * RCT(0, 2)); \
    loss = loss + (YN(2) * RCT(0, 3)); \
    prod = prod + (YN(3) * (YN(2) * RCT(0, 4))); \
    loss = loss + RCT(0, 5); \
    prod = prod + (YO(6) * RCT(0, 6)); \
    loss = loss + (YN(3) * RCT(0, 7)); \
    prod = prod + (YN(2) * (YO(6) * RCT(0, 8))); \
    loss = loss + (YO(4) * RCT(0, 9)); \
    prod = prod + (YN(2) * (YO(6) * RCT(0, 8))); \
    loss = loss + (YO(4) * RCT(0, 9)); \
    prod = prod + (YN(3) * (YO(6) * RCT(0, 10))); \
    loss = loss + (YN(1) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 88); \
    TM_LD(0, 1, 90); \
    TM_LD(0, 2, 104); \
    TM_LD(0, 3, 106); \
    TM_LD(0, 4, 114); \
    TM_LD(0, 5, 112); \
    TM_LD(0, 6, 132); \
    TM_LD(0, 7, 134); \
    TM_LD(0, 8, 138); \
    TM_LD(0, 9, 136); \
    TM_LD(0, 10, 154); \
    TM_LD(0, 11, 152); \
    prod = prod + (YN(1) * (YO(5) * RCT(1, 0))); \
    loss = loss + (YO(6) * RCT(1, 1)); \
    prod = prod + (YO(7) * RCT(1, 2)); \
    loss = loss + (YO(4) * RCT(1, 3)); \
    prod = prod + (YO(7) * RCT(1, 2)); \
    loss = loss + (YO(4) * RCT(1, 3)); \
    prod = prod + (YN(2) * (YO(7) * RCT(1, 4))); \
    loss = loss + (YO(5) * RCT(1, 5)); \
    prod = prod + ((YO(5) * YO(6)) * RCT(1, 6)); \
    loss = loss + (YO(7) * RCT(1, 7)); \
    prod = prod + (YN(3) * (YO(7) * RCT(1, 8))); \
    loss = loss + (YO(6) * RCT(1, 9)); \
    prod = prod + (YN(2) * (YO(9) * RCT(1, 10))); \
    loss = loss + (YO(8) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 156); \
    TM_LD(1, 1, 158); \
    TM_LD(1, 2, 178); \
    TM_LD(1, 3, 176); \
    TM_LD(1, 4, 188); \
    TM_LD(1, 5, 190); \
    TM_LD(1, 6, 192); \
    TM_LD(1, 7, 194); \
    TM_LD(1, 8, 218); \
    TM_LD(1, 9, 216); \
    TM_LD(1, 10, 234); \
    TM_LD(1, 11, 232); \
    prod = prod + ((YO(8) * YO(6)) * RCT(0, 0)); \
    loss = loss + (YO(9) * RCT(0, 1)); \
    prod = prod + (YN(3) * (YO(10) * RCT(0, 2))); \
    loss = loss + (YO(8) * RCT(0, 3)); \
    prod = prod + ((YO(8) * YO(5)) * RCT(0, 4)); \
    loss = loss + (YO(10) * RCT(0, 5)); \
    prod = prod + (YN(3) * (YO(11) * RCT(0, 6))); \
    loss = loss + (YO(10) * RCT(0, 7)); \
    prod = prod + ((YO(10) * YO(5)) * RCT(0, 8)); \
    loss = loss + (YO(11) * RCT(0, 9)); \
    prod = prod + ((YO(5) * YO(13)) * RCT(0, 10)); \
    loss = loss + (YO(12) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 238); \
    TM_LD(0, 1, 236); \
    TM_LD(0, 2, 274); \
    TM_LD(0, 3, 272); \
    TM_LD(0, 4, 276); \
    TM_LD(0, 5, 278); \
    TM_LD(0, 6, 292); \
    TM_LD(0, 7, 294); \
    TM_LD(0, 8, 298); \
    TM_LD(0, 9, 296); \
    TM_LD(0, 10, 316); \
    TM_LD(0, 11, 318); \
    prod = prod + (YN(3) * (YO(12) * RCT(1, 0))); \
    loss = loss + (YO(13) * RCT(1, 1)); \
    prod = prod + ((YO(15) * YO(5)) * RCT(1, 2)); \
    loss = loss + (YO(13) * RCT(1, 3)); \
    prod = prod + ((YO(13) * YO(6)) * RCT(1, 4)); \
    loss = loss + (YO(17) * RCT(1, 5)); \
    prod = prod + (YN(1) * (YO(13) * RCT(1, 6))); \
    loss = loss + (YO(11) * RCT(1, 7)); \
    prod = prod + (YN(2) * (YO(11) * RCT(1, 8))); \
    loss = loss + (YO(15) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(15) * RCS(0))); \
    loss = loss + ((YO(8) * YN(2)) * RCS(1)); \
    prod = prod + (YN(2) * (YO(11) * RCT(1, 10))); \
    loss = loss + (YO(14) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 338); \
    TM_LD(1, 1, 336); \
    TM_LD(1, 2, 356); \
    TM_LD(1, 3, 358); \
    TM_LD(1, 4, 392); \
    TM_LD(1, 5, 394); \
    TM_LD(1, 6, 422); \
    TM_LD(1, 7, 420); \
    TM_LD(1, 8, 8); \
    TM_LD(1, 9, 10); \
    TM_LD(1, 10, 14); \
    TM_LD(1, 11, 12); \
    prod = prod + ((YO(20) * YO(5)) * RCT(0, 0)); \
    loss = loss + (YO(14) * RCT(0, 1)); \
    prod = prod + (YN(1) * (YO(14) * RCS(4))); \
    loss = loss + ((YO(8) * YN(2)) * RCS(5)); \
    prod = prod + ((YO(11) * YO(5)) * RCT(0, 2)); \
    loss = loss + (YO(17) * RCT(0, 3)); \
    prod = prod + (YN(3) * (YO(17) * RCT(0, 4))); \
    loss = loss + (YO(11) * RCT(0, 5)); \
    prod = prod + (YN(3) * (YO(19) * RCT(0, 6))); \
    loss = loss + (YO(18) * RCT(0, 7)); \
    prod = prod + ((YO(18) * YO(5)) * RCT(0, 8)); \
    loss = loss + (YO(19) * RCT(0, 9)); \
    prod = prod + (YN(3) * (YO(18) * RCT(0, 10))); \
    loss = loss + (YO(16) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 20); \
    TM_LD(0, 1, 22); \
    TM_LD(0, 2, 48); \
    TM_LD(0, 3, 50); \
    TM_LD(0, 4, 56); \
    TM_LD(0, 5, 58); \
    TM_LD(0, 6, 72); \
    TM_LD(0, 7, 74); \
    TM_LD(0, 8, 76); \
    TM_LD(0, 9, 78); \
    TM_LD(0, 10, 112); \
    TM_LD(0, 11, 114); \
    prod = prod + ((YO(22) * YO(5)) * RCT(1, 0)); \
    loss = loss + (YO(16) * RCT(1, 1)); \
    prod = prod + ((YO(16) * YO(6)) * RCT(1, 2)); \
    loss = loss + (YO(24) * RCT(1, 3)); \
    prod = prod + (YN(2) * (YO(25) * RCS(19))); \
    loss = loss + (YO(21) * RCS(18)); \
    prod = prod + ((YO(27) * YO(5)) * RCS(21)); \
    loss = loss + (YO(21) * RCS(20)); \
    prod = prod + (YN(3) * (YO(25) * RCS(26))); \
    loss = loss + (YO(26) * RCS(27)); \
    prod = prod + (YN(2) * ((YO(10) * YO(8)) * RCS(33))); \
    loss = loss + (YO(26) * RCS(32)); \
    prod = prod + (YN(1) * (YO(26) * RCS(36))); \
    loss = loss + ((YO(8) * YO(8)) * RCS(37)); \
    prod = prod + (YN(2) * (YO(26) * RCS(41))); \
    loss = loss + (YO(27) * RCS(40)); \
    prod = prod + (YN(2) * (YO(28) * RCS(52))); \
    loss = loss + (YO(13) * RCS(53)); \
    prod = prod + ((YO(11) * YO(5)) * RCS(55)); \
    loss = loss + (YO(28) * RCS(54)); \
    prod = prod + ((YO(28) * YO(8)) * RCS(59)); \
    loss = loss + (YO(25) * RCS(58)); \
    prod = prod + ((YO(28) * YO(5)) * RCS(61)); \
    loss = loss + (YO(29) * RCS(60)); \
    prod = prod + ((YO(17) * YO(5)) * RCS(63)); \
    loss = loss + (YO(29) * RCS(62)); \
    prod = prod + (YN(3) * (YO(29) * RCS(68))); \
    loss = loss + (YO(28) * RCS(69)); \
    prod = prod + (YO(29) * RCT(1, 4)); \
    loss = loss + (YO(13) * RCT(1, 5)); \
    prod = prod + ((YO(25) * YO(5)) * RCS(81)); \
    loss = loss + (YO(23) * RCS(80)); \
    prod = prod + (YN(1) * (YO(23) * RCS(82))); \
    loss = loss + ((YO(11) * YO(8)) * RCS(83)); \
    prod = prod + ((YO(23) * YO(6)) * RCS(86)); \
    loss = loss + ((YO(11) * YO(10)) * RCS(87)); \
    prod = prod + ((YO(34) * YO(5)) * RCS(91)); \
    loss = loss + (YO(31) * RCS(90)); \
    prod = prod + ((YO(23) * YO(5)) * RCS(93)); \
    loss = loss + (YO(31) * RCS(92)); \
    prod = prod + (YN(3) * (YO(31) * RCS(94))); \
    loss = loss + (YO(34) * RCS(95)); \
    prod = prod + (YN(3) * (YO(31) * RCS(96))); \
    loss = loss + (YO(23) * RCS(97)); \
    prod = prod + ((YO(33) * YO(5)) * RCS(113)); \
    loss = loss + (YO(30) * RCS(112)); \
    prod = prod + ((YO(32) * YO(5)) * RCS(115)); \
    loss = loss + (YO(30) * RCS(114)); \
    prod = prod + ((YO(35) * YO(5)) * RCS(117)); \
    loss = loss + (YO(30) * RCS(116)); \
    prod = prod + (YN(3) * (YO(30) * RCS(124))); \
    loss = loss + (YO(33) * RCS(125)); \
    prod = prod + (YN(3) * (YO(30) * RCS(126))); \
    loss = loss + (YO(32) * RCS(127)); \
    prod = prod + (YN(3) * (YO(30) * RCS(128))); \
    loss = loss + (YO(35) * RCS(129)); \
    prod = prod + (YO(33) * RCT(1, 6)); \
    loss = loss + (YO(16) * RCT(1, 7)); \
    prod = prod + ((YO(18) * YO(6)) * RCS(142)); \
    loss = loss + (YO(35) * RCS(143)); \
    prod = prod + ((YO(31) * YO(5)) * RCS(153)); \
    loss = loss + (YO(35) * RCS(152)); \
    prod = prod + (YN(3) * (YO(32) * RCS(156))); \
    loss = loss + (YO(31) * RCS(157)); \
    prod = prod + ((YO(32) * YO(6)) * RCS(162)); \
    loss = loss + ((YO(31) * YO(4)) * RCS(163)); \
    prod = prod + ((YO(32) * YO(6)) * RCS(162)); \
    loss = loss + ((YO(31) * YO(4)) * RCS(163)); \
    prod = prod + ((YO(31) * YO(5)) * RCS(165)); \
    loss = loss + (YO(32) * RCS(164)); \
    prod = prod + ((YO(37) * YO(5)) * RCS(175)); \
    loss = loss + (YO(36) * RCS(174)); \
    prod = prod + ((YO(36) * YO(5)) * RCS(185)); \
    loss = loss + (YO(38) * RCS(184)); \
    prod = prod + ((YO(37) * YO(6)) * RCS(188)); \
    loss = loss + ((YO(8) * YO(22)) * RCS(189)); \
    prod = prod + ((YO(38) * YO(5)) * RCS(195)); \
    loss = loss + (YO(39) * RCS(194)); \
    prod = prod + ((YO(38) * YO(6)) * RCS(202)); \
    loss = loss + ((YO(22) * YO(11)) * RCS(203)); \
    prod = prod + (YN(3) * (YO(40) * RCS(216))); \
    loss = loss + (YO(41) * RCS(217)); \
    prod = prod + (YN(3) * (YO(40) * RCS(218))); \
    loss = loss + (YO(42) * RCS(219)); \
    prod = prod + ((YO(42) * YO(5)) * RCS(221)); \
    loss = loss + (YO(40) * RCS(220)); \
    prod = prod + ((YO(41) * YO(5)) * RCS(223)); \
    loss = loss + (YO(40) * RCS(222)); \
    prod = prod + (YN(2) * ((YO(44) * YO(38)) * RCS(239))); \
    loss = loss + (YO(43) * RCS(238)); \
    prod = prod + (((YO(5) * YO(48)) * YO(18)) * RCS(257)); \
    loss = loss + (YO(46) * RCS(256)); \
    prod = prod + 0.0; \
    loss = loss + (YO(46) * RCS(258)); \
    prod = prod + 0.0; \
    loss = loss + (YO(46) * RCS(259)); \
    prod = prod + 0.0; \
    loss = loss + (YO(46) * RCS(260)); \
    prod = prod + (((YO(5) * YO(39)) * YO(22)) * RCS(262)); \
    loss = loss + (YO(48) * RCS(261)); \
    prod = prod + (YN(2) * ((YO(5) * YO(43)) * RCS(280))); \
    loss = loss + (YO(47) * RCS(279)); \
    loss = loss + SOUR(3); \
    rhs1 = rho * Y0S(0) + dt * WM(4) * (prod + extra); \
    rhs2 = -(dt * WM(4) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(4) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(4) - fnew); \
    UC_UPDATE_TAIL(4); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 6); \
    prod = (YN(4) * (YN(0) * RCT(1, 8))); \
    extra = (1.0 * (YN(4) * (YO(46) * RCS(258)))); \
    loss = (YN(2) * RCT(1, 9)); \
    prod = prod + (YN(4) * (YOS(1) * RCT(1, 10))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(259)))); \
    loss = loss + (YN(3) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 136); \
    TM_LD(1, 1, 138); \
    TM_LD(1, 2, 152); \
    TM_LD(1, 3, 154); \
    TM_LD(1, 4, 176); \
    TM_LD(1, 5, 178); \
    TM_LD(1, 6, 236); \
    TM_LD(1, 7, 238); \
    TM_LD(1, 8, 258); \
    TM_LD(1, 9, 256); \
    TM_LD(1, 10, 268); \
    TM_LD(1, 11, 270); \
    prod = prod + (YN(4) * (YN(2) * RCT(0, 0))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    loss = loss + RCT(0, 1); \
    prod = prod + (YN(2) * (YO(6) * RCT(0, 2))); \
    loss = loss + (YN(3) * RCT(0, 3)); \
    prod = prod + (YN(4) * (YO(6) * RCT(0, 4))); \
    loss = loss + (YN(1) * RCT(0, 5)); \
    prod = prod + (YN(2) * (YO(7) * RCT(0, 6))); \
    loss = loss + (YN(4) * RCT(0, 7)); \
    prod = prod + (YN(4) * (YO(7) * RCT(0, 8))); \
    loss = loss + (YO(6) * RCT(0, 9)); \
    prod = prod + (YN(4) * (YO(10) * RCT(0, 10))); \
    loss = loss + (YO(8) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 272); \
    TM_LD(0, 1, 274); \
    TM_LD(0, 2, 296); \
    TM_LD(0, 3, 298); \
    TM_LD(0, 4, 336); \
    TM_LD(0, 5, 338); \
    TM_LD(0, 6, 416); \
    TM_LD(0, 7, 418); \
    TM_LD(0, 8, 32); \
    TM_LD(0, 9, 34); \
    TM_LD(0, 10, 36); \
    TM_LD(0, 11, 38); \
    prod = prod + (YN(4) * (YO(11) * RCT(1, 0))); \
    loss = loss + (YO(10) * RCT(1, 1)); \
    prod = prod + (YN(4) * (YO(12) * RCT(1, 2))); \
    loss = loss + (YO(13) * RCT(1, 3)); \
    prod = prod + (YN(4) * (YO(13) * RCT(1, 4))); \
    loss = loss + (YO(15) * RCT(1, 5)); \
    prod = prod + (YN(4) * (YO(14) * RCT(1, 6))); \
    loss = loss + (YO(20) * RCT(1, 7)); \
    prod = prod + (YN(2) * (YO(11) * RCT(1, 8))); \
    loss = loss + (YO(20) * RCT(1, 9)); \
    prod = prod + (YN(2) * (YO(17) * RCT(1, 10))); \
    loss = loss + (YO(15) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 42); \
    TM_LD(1, 1, 40); \
    TM_LD(1, 2, 46); \
    TM_LD(1, 3, 44); \
    TM_LD(1, 4, 50); \
    TM_LD(1, 5, 48); \
    TM_LD(1, 6, 54); \
    TM_LD(1, 7, 52); \
    TM_LD(1, 8, 58); \
    TM_LD(1, 9, 56); \
    TM_LD(1, 10, 66); \
    TM_LD(1, 11, 64); \
    prod = prod + (YN(4) * (YO(17) * RCT(0, 0))); \
    loss = loss + (YO(11) * RCT(0, 1)); \
    prod = prod + (YN(4) * (YO(19) * RCT(0, 2))); \
    loss = loss + (YO(18) * RCT(0, 3)); \
    prod = prod + (YN(4) * (YO(16) * RCT(0, 4))); \
    loss = loss + (YO(22) * RCT(0, 5)); \
    prod = prod + (YN(4) * (YO(21) * RCS(20))); \
    loss = loss + (YO(27) * RCS(21)); \
    prod = prod + (YN(4) * (YO(28) * RCS(54))); \
    loss = loss + (YO(11) * RCS(55)); \
    prod = prod + (YN(4) * (YO(29) * RCS(60))); \
    loss = loss + (YO(28) * RCS(61)); \
    prod = prod + (YN(4) * (YO(29) * RCS(62))); \
    loss = loss + (YO(17) * RCS(63)); \
    prod = prod + (YN(4) * (YO(23) * RCS(80))); \
    loss = loss + (YO(25) * RCS(81)); \
    prod = prod + (YN(4) * (YO(31) * RCS(90))); \
    loss = loss + (YO(34) * RCS(91)); \
    prod = prod + (YN(4) * (YO(31) * RCS(92))); \
    loss = loss + (YO(23) * RCS(93)); \
    prod = prod + (YO(30) * RCT(0, 6)); \
    loss = loss + (YO(16) * RCT(0, 7)); \
    prod = prod + (YN(4) * (YO(30) * RCS(112))); \
    loss = loss + (YO(33) * RCS(113)); \
    prod = prod + (YN(4) * (YO(30) * RCS(114))); \
    loss = loss + (YO(32) * RCS(115)); \
    prod = prod + (YN(4) * (YO(30) * RCS(116))); \
    loss = loss + (YO(35) * RCS(117)); \
    prod = prod + (YN(2) * (YO(35) * RCS(150))); \
    loss = loss + (YO(16) * RCS(151)); \
    prod = prod + (YN(4) * (YO(35) * RCS(152))); \
    loss = loss + (YO(31) * RCS(153)); \
    prod = prod + (YN(2) * (YO(32) * RCS(158))); \
    loss = loss + (YO(16) * RCS(159)); \
    prod = prod + (YN(4) * (YO(32) * RCS(164))); \
    loss = loss + (YO(31) * RCS(165)); \
    prod = prod + (YN(4) * (YO(36) * RCS(174))); \
    loss = loss + (YO(37) * RCS(175)); \
    prod = prod + (YN(4) * (YO(38) * RCS(184))); \
    loss = loss + (YO(36) * RCS(185)); \
    prod = prod + (YN(4) * (YO(39) * RCS(194))); \
    loss = loss + (YO(38) * RCS(195)); \
    prod = prod + (YN(4) * (YO(40) * RCS(220))); \
    loss = loss + (YO(42) * RCS(221)); \
    prod = prod + (YN(4) * (YO(40) * RCS(222))); \
    loss = loss + (YO(41) * RCS(223)); \
    prod = prod + (YN(4) * (YO(46) * RCS(256))); \
    loss = loss + ((YO(48) * YO(18)) * RCS(257)); \
    prod = prod + (YN(4) * (YO(48) * RCS(261))); \
    loss = loss + ((YO(39) * YO(22)) * RCS(262)); \
    prod = prod + (YN(4) * (YO(47) * RCS(279))); \
    loss = loss + ((YO(43) * YN(2)) * RCS(280)); \
    rhs1 = rho * Y0S(1) + dt * WM(5) * (prod + extra); \
    rhs2 = -(dt * WM(5) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(5) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(5) - fnew); \
    UC_UPDATE_TAIL(5); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 7); \
    prod = (YN(4) * (YN(3) * RCT(0, 8))); \
    extra = 0.0; \
    loss = RCT(0, 9); \
    prod = prod + (YN(2) * (YN(1) * RCT(0, 10))); \
    loss = loss + RCT(0, 11); \
    TM_WAIT(1); \
    TM_LD(0, 0, 68); \
    TM_LD(0, 1, 70); \
    TM_LD(0, 2, 76); \
    TM_LD(0, 3, 78); \
    TM_LD(0, 4, 80); \
    TM_LD(0, 5, 82); \
    TM_LD(0, 6, 90); \
    TM_LD(0, 7, 88); \
    TM_LD(0, 8, 116); \
    TM_LD(0, 9, 118); \
    TM_LD(0, 10, 140); \
    TM_LD(0, 11, 142); \
    prod = prod + (YN(4) * (YOS(1) * RCT(1, 0))); \
    loss = loss + (YN(2) * RCT(1, 1)); \
    prod = prod + (YN(1) * (YN(0) * RCT(1, 2))); \
    loss = loss + (YN(2) * RCT(1, 3)); \
    prod = prod + (YN(5) * (YN(3) * RCT(1, 4))); \
    loss = loss + (YN(2) * RCT(1, 5)); \
    prod = prod + (YN(4) * (YN(1) * RCT(1, 6))); \
    loss = loss + (YN(3) * RCT(1, 7)); \
    prod = prod + (YN(5) * (YN(1) * RCT(1, 8))); \
    loss = loss + (YN(4) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(7) * RCT(1, 10))); \
    loss = loss + (YO(6) * RCT(1, 11)); \
    prod = prod + (YN(1) * (YO(7) * RCT(1, 10))); \
    loss = loss + (YO(6) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 146); \
    TM_LD(1, 1, 144); \
    TM_LD(1, 2, 160); \
    TM_LD(1, 3, 162); \
    TM_LD(1, 4, 166); \
    TM_LD(1, 5, 164); \
    TM_LD(1, 6, 190); \
    TM_LD(1, 7, 188); \
    TM_LD(1, 8, 280); \
    TM_LD(1, 9, 282); \
    TM_LD(1, 10, 310); \
    TM_LD(1, 11, 308); \
    prod = prod + (YN(2) * (YO(7) * RCT(0, 0))); \
    loss = loss + (YN(0) * RCT(0, 1)); \
    prod = prod + (YN(4) * (YO(7) * RCT(0, 2))); \
    loss = loss + (YN(5) * RCT(0, 3)); \
    prod = prod + (YN(3) * (YO(7) * RCT(0, 4))); \
    loss = loss + (YN(4) * RCT(0, 5)); \
    prod = prod + (YN(4) * (YO(9) * RCT(0, 6))); \
    loss = loss + (YO(8) * RCT(0, 7)); \
    prod = prod + (YN(1) * (YO(10) * RCT(0, 8))); \
    loss = loss + (YO(8) * RCT(0, 9)); \
    prod = prod + (YN(1) * (YO(11) * RCT(0, 10))); \
    loss = loss + (YO(10) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 324); \
    TM_LD(0, 1, 326); \
    TM_LD(0, 2, 352); \
    TM_LD(0, 3, 354); \
    TM_LD(0, 4, 358); \
    TM_LD(0, 5, 356); \
    TM_LD(0, 6, 60); \
    TM_LD(0, 7, 62); \
    TM_LD(0, 8, 64); \
    TM_LD(0, 9, 66); \
    TM_LD(0, 10, 70); \
    TM_LD(0, 11, 68); \
    prod = prod + ((YO(10) * YO(7)) * RCT(1, 0)); \
    loss = loss + (YO(11) * RCT(1, 1)); \
    prod = prod + (YN(1) * (YO(12) * RCT(1, 2))); \
    loss = loss + (YO(13) * RCT(1, 3)); \
    prod = prod + ((YO(13) * YO(7)) * RCT(1, 4)); \
    loss = loss + (YO(12) * RCT(1, 5)); \
    prod = prod + (YN(4) * (YO(17) * RCT(1, 6))); \
    loss = loss + (YO(13) * RCT(1, 7)); \
    prod = prod + (YN(1) * (YO(17) * RCT(1, 8))); \
    loss = loss + (YO(11) * RCT(1, 9)); \
    prod = prod + ((YO(18) * YO(7)) * RCT(1, 10)); \
    loss = loss + (YO(19) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 74); \
    TM_LD(1, 1, 72); \
    TM_LD(1, 2, 78); \
    TM_LD(1, 3, 76); \
    TM_LD(1, 4, 82); \
    TM_LD(1, 5, 80); \
    TM_LD(1, 6, 144); \
    TM_LD(1, 7, 146); \
    TM_LD(1, 8, 164); \
    TM_LD(1, 9, 166); \
    TM_LD(1, 10, 308); \
    TM_LD(1, 11, 310); \
    prod = prod + (YN(1) * (YO(18) * RCT(0, 0))); \
    loss = loss + (YO(16) * RCT(0, 1)); \
    prod = prod + (YN(1) * (YO(16) * RCT(0, 2))); \
    loss = loss + (YO(22) * RCT(0, 3)); \
    prod = prod + (YN(4) * (YO(24) * RCT(0, 4))); \
    loss = loss + (YO(16) * RCT(0, 5)); \
    prod = prod + (((YO(13) * YO(8)) * YO(7)) * RCS(9)); \
    loss = loss + (YO(24) * RCS(8)); \
    prod = prod + (YN(1) * (YO(22) * RCS(10))); \
    loss = loss + (YO(21) * RCS(11)); \
    prod = prod + (YN(1) * (YO(28) * RCS(56))); \
    loss = loss + (YO(11) * RCS(57)); \
    prod = prod + ((YO(28) * YO(7)) * RCS(71)); \
    loss = loss + (YO(29) * RCS(70)); \
    prod = prod + (YN(1) * (YO(29) * RCS(72))); \
    loss = loss + (YO(28) * RCS(73)); \
    prod = prod + (YN(4) * ((YO(11) * YO(10)) * RCS(87))); \
    loss = loss + (YO(23) * RCS(86)); \
    prod = prod + (YN(1) * (YO(31) * RCS(89))); \
    loss = loss + (YO(23) * RCS(88)); \
    prod = prod + ((YO(34) * YO(7)) * RCS(107)); \
    loss = loss + (YO(31) * RCS(106)); \
    prod = prod + ((YO(23) * YO(7)) * RCS(109)); \
    loss = loss + (YO(31) * RCS(108)); \
    prod = prod + (YN(1) * (YO(31) * RCS(110))); \
    loss = loss + (YO(34) * RCS(111)); \
    prod = prod + ((YO(32) * YO(7)) * RCS(137)); \
    loss = loss + (YO(30) * RCS(136)); \
    prod = prod + ((YO(33) * YO(7)) * RCS(139)); \
    loss = loss + (YO(30) * RCS(138)); \
    prod = prod + ((YO(35) * YO(7)) * RCS(141)); \
    loss = loss + (YO(30) * RCS(140)); \
    prod = prod + (YN(4) * (YO(35) * RCS(143))); \
    loss = loss + (YO(18) * RCS(142)); \
    prod = prod + (YN(1) * (YO(35) * RCS(144))); \
    loss = loss + (YO(31) * RCS(145)); \
    prod = prod + (YN(1) * (YO(32) * RCS(154))); \
    loss = loss + (YO(31) * RCS(155)); \
    prod = prod + (YN(4) * ((YO(31) * YOS(1)) * RCS(163))); \
    loss = loss + (YO(32) * RCS(162)); \
    prod = prod + (YN(1) * (YO(36) * RCS(173))); \
    loss = loss + (YO(37) * RCS(172)); \
    prod = prod + (YN(1) * (YO(38) * RCS(180))); \
    loss = loss + (YO(36) * RCS(181)); \
    prod = prod + (YN(4) * ((YO(8) * YO(22)) * RCS(189))); \
    loss = loss + (YO(37) * RCS(188)); \
    prod = prod + (YN(1) * (YO(39) * RCS(201))); \
    loss = loss + (YO(38) * RCS(200)); \
    prod = prod + (YN(4) * ((YO(22) * YO(11)) * RCS(203))); \
    loss = loss + (YO(38) * RCS(202)); \
    prod = prod + (YN(1) * (YO(40) * RCS(208))); \
    loss = loss + (YO(41) * RCS(209)); \
    prod = prod + (YN(1) * (YO(40) * RCS(210))); \
    loss = loss + (YO(42) * RCS(211)); \
    prod = prod + ((YO(41) * YO(7)) * RCS(225)); \
    loss = loss + (YO(40) * RCS(224)); \
    prod = prod + ((YO(42) * YO(7)) * RCS(227)); \
    loss = loss + (YO(40) * RCS(226)); \
    prod = prod + (YN(1) * (YO(41) * RCS(228))); \
    loss = loss + (YO(39) * RCS(229)); \
    prod = prod + (YN(1) * (YO(42) * RCS(230))); \
    loss = loss + (YO(39) * RCS(231)); \
    prod = prod + (YN(1) * (YO(45) * RCS(242))); \
    loss = loss + ((YO(21) * YO(38)) * RCS(243)); \
    prod = prod + (YN(1) * (YO(45) * RCS(244))); \
    loss = loss + ((YO(22) * YO(36)) * RCS(245)); \
    prod = prod + (((YO(21) * YO(38)) * YO(7)) * RCS(247)); \
    loss = loss + (YO(45) * RCS(246)); \
    prod = prod + (((YO(22) * YO(36)) * YO(7)) * RCS(249)); \
    loss = loss + (YO(45) * RCS(248)); \
    rhs1 = rho * Y0S(0) + dt * WM(6) * (prod + extra); \
    rhs2 = -(dt * WM(6) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(6) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(6) - fnew); \
    UC_UPDATE_TAIL(6); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 8); \
    prod = (YN(4) * (YOS(1) * RCT(0, 6))); \
    extra = 0.0; \
    loss = RCT(0, 7); \
    prod = prod + (YN(6) * (YOS(2) * RCT(0, 8))); \
    loss = loss + (YN(1) * RCT(0, 9)); \
    prod = prod + (YN(6) * (YN(0) * RCT(0, 10))); \
    loss = loss + (YN(2) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 86); \
    TM_LD(0, 1, 84); \
    TM_LD(0, 2, 90); \
    TM_LD(0, 3, 88); \
    TM_LD(0, 4, 94); \
    TM_LD(0, 5, 92); \
    TM_LD(0, 6, 96); \
    TM_LD(0, 7, 98); \
    TM_LD(0, 8, 100); \
    TM_LD(0, 9, 102); \
    TM_LD(0, 10, 104); \
    TM_LD(0, 11, 106); \
    prod = prod + (YN(5) * (YN(4) * RCT(1, 0))); \
    loss = loss + (YN(2) * RCT(1, 1)); \
    prod = prod + (YN(6) * (YN(5) * RCT(1, 2))); \
    loss = loss + (YN(4) * RCT(1, 3)); \
    prod = prod + (YN(6) * (YN(4) * RCT(1, 4))); \
    loss = loss + (YN(3) * RCT(1, 5)); \
    prod = prod + (YN(6) * (YO(11) * RCT(1, 6))); \
    loss = loss + (YO(10) * RCT(1, 7)); \
    prod = prod + (YN(6) * (YO(12) * RCT(1, 8))); \
    loss = loss + (YO(13) * RCT(1, 9)); \
    prod = prod + (YN(6) * (YO(19) * RCT(1, 10))); \
    loss = loss + (YO(18) * RCT(1, 11)); \
    prod = prod + (YN(6) * (YO(24) * RCS(8))); \
    loss = loss + ((YO(13) * YO(8)) * RCS(9)); \
    prod = prod + (YN(6) * (YO(29) * RCS(70))); \
    loss = loss + (YO(28) * RCS(71)); \
    prod = prod + (YN(6) * (YO(31) * RCS(106))); \
    loss = loss + (YO(34) * RCS(107)); \
    prod = prod + (YN(6) * (YO(31) * RCS(108))); \
    loss = loss + (YO(23) * RCS(109)); \
    prod = prod + (YN(6) * (YO(30) * RCS(136))); \
    loss = loss + (YO(32) * RCS(137)); \
    prod = prod + (YN(6) * (YO(30) * RCS(138))); \
    loss = loss + (YO(33) * RCS(139)); \
    prod = prod + (YN(6) * (YO(30) * RCS(140))); \
    loss = loss + (YO(35) * RCS(141)); \
    prod = prod + (YN(6) * (YO(40) * RCS(224))); \
    loss = loss + (YO(41) * RCS(225)); \
    prod = prod + (YN(6) * (YO(40) * RCS(226))); \
    loss = loss + (YO(42) * RCS(227)); \
    prod = prod + (YN(6) * (YO(45) * RCS(246))); \
    loss = loss + ((YO(21) * YO(38)) * RCS(247)); \
    prod = prod + (YN(6) * (YO(45) * RCS(248))); \
    loss = loss + ((YO(22) * YO(36)) * RCS(249)); \
    rhs1 = rho * Y0S(1) + dt * WM(7) * (prod + extra); \
    rhs2 = -(dt * WM(7) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(7) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(7) - fnew); \
    UC_UPDATE_TAIL(7); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 9); \
    TM_WAIT(0); \
    TM_LD(1, 0, 112); \
    TM_LD(1, 1, 114); \
    TM_LD(1, 2, 116); \
    TM_LD(1, 3, 118); \
    TM_LD(1, 4, 120); \
    TM_LD(1, 5, 122); \
    TM_LD(1, 6, 220); \
    TM_LD(1, 7, 222); \
    TM_LD(1, 8, 240); \
    TM_LD(1, 9, 242); \
    TM_LD(1, 10, 248); \
    TM_LD(1, 11, 250); \
    prod = (YN(2) * (YO(9) * RCT(0, 0))); \
    extra = 0.0; \
    loss = (YN(4) * RCT(0, 1)); \
    prod = prod + (YN(4) * (YO(9) * RCT(0, 2))); \
    loss = loss + (YN(6) * RCT(0, 3)); \
    prod = prod + (YN(3) * (YO(9) * RCT(0, 4))); \
    loss = loss + (YN(1) * RCT(0, 5)); \
    prod = prod + (YO(10) * RCT(0, 6)); \
    loss = loss + (YN(2) * RCT(0, 7)); \
    prod = prod + (YN(2) * (YO(10) * RCT(0, 8))); \
    loss = loss + (YN(0) * RCT(0, 9)); \
    prod = prod + (YN(3) * (YO(10) * RCT(0, 10))); \
    loss = loss + (YN(4) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 260); \
    TM_LD(0, 1, 262); \
    TM_LD(0, 2, 400); \
    TM_LD(0, 3, 402); \
    TM_LD(0, 4, 408); \
    TM_LD(0, 5, 410); \
    TM_LD(0, 6, 84); \
    TM_LD(0, 7, 86); \
    TM_LD(0, 8, 88); \
    TM_LD(0, 9, 90); \
    TM_LD(0, 10, 92); \
    TM_LD(0, 11, 94); \
    prod = prod + (YN(4) * (YO(10) * RCT(1, 0))); \
    loss = loss + (YN(5) * RCT(1, 1)); \
    prod = prod + (YN(1) * (YO(10) * RCT(1, 2))); \
    loss = loss + (YN(6) * RCT(1, 3)); \
    prod = prod + ((YO(10) * YO(13)) * RCT(1, 4)); \
    loss = loss + (YO(12) * RCT(1, 5)); \
    prod = prod + (YN(1) * (YO(15) * RCS(0))); \
    loss = loss + ((YN(4) * YN(2)) * RCS(1)); \
    prod = prod + ((YO(15) * YO(9)) * RCT(1, 6)); \
    loss = loss + (YO(11) * RCT(1, 7)); \
    prod = prod + (YN(3) * (YO(14) * RCS(2))); \
    loss = loss + ((YN(2) * YN(2)) * RCS(3)); \
    prod = prod + (YN(3) * (YO(14) * RCT(1, 8))); \
    loss = loss + (YN(0) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(14) * RCS(4))); \
    loss = loss + ((YN(4) * YN(2)) * RCS(5)); \
    prod = prod + (YN(3) * (YO(20) * RCT(1, 10))); \
    loss = loss + (YN(2) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 108); \
    TM_LD(1, 1, 110); \
    TM_LD(1, 2, 222); \
    TM_LD(1, 3, 220); \
    TM_LD(1, 4, 244); \
    TM_LD(1, 5, 246); \
    TM_LD(1, 6, 262); \
    TM_LD(1, 7, 260); \
    TM_LD(1, 8, 98); \
    TM_LD(1, 9, 96); \
    TM_LD(1, 10, 102); \
    TM_LD(1, 11, 100); \
    prod = prod + ((YO(20) * YO(9)) * RCT(0, 0)); \
    loss = loss + (YO(10) * RCT(0, 1)); \
    prod = prod + (YN(6) * (YO(24) * RCS(8))); \
    loss = loss + ((YO(13) * YN(7)) * RCS(9)); \
    prod = prod + (YN(3) * (YO(21) * RCS(14))); \
    loss = loss + (YO(14) * RCS(15)); \
    prod = prod + (YN(1) * (YO(21) * RCS(16))); \
    loss = loss + (YO(11) * RCS(17)); \
    prod = prod + (YN(2) * (YO(25) * RCS(22))); \
    loss = loss + (YO(13) * RCS(23)); \
    prod = prod + ((YO(25) * YO(13)) * RCS(28)); \
    loss = loss + (YO(18) * RCS(29)); \
    prod = prod + (YN(2) * (YO(26) * RCS(30))); \
    loss = loss + (YO(15) * RCS(31)); \
    prod = prod + (YN(4) * (YO(26) * RCS(32))); \
    loss = loss + ((YO(10) * YN(2)) * RCS(33)); \
    prod = prod + (YN(3) * (YO(26) * RCS(34))); \
    loss = loss + ((YO(8) * YN(2)) * RCS(35)); \
    prod = prod + (YN(3) * (YO(26) * RCS(34))); \
    loss = loss + ((YO(8) * YN(2)) * RCS(35)); \
    prod = prod + (YN(1) * (YO(26) * RCS(36))); \
    loss = loss + ((YO(8) * YN(4)) * RCS(37)); \
    prod = prod + (YN(1) * (YO(26) * RCS(36))); \
    loss = loss + ((YO(8) * YN(4)) * RCS(37)); \
    prod = prod + (YN(1) * (YO(26) * RCS(38))); \
    loss = loss + ((YO(9) * YN(2)) * RCS(39)); \
    prod = prod + (YN(3) * (YO(27) * RCS(42))); \
    loss = loss + (YO(20) * RCS(43)); \
    prod = prod + (YN(1) * (YO(27) * RCS(48))); \
    loss = loss + (YO(10) * RCS(49)); \
    prod = prod + (YN(4) * (YO(25) * RCS(58))); \
    loss = loss + (YO(28) * RCS(59)); \
    prod = prod + (YN(1) * (YO(23) * RCS(82))); \
    loss = loss + ((YO(11) * YN(4)) * RCS(83)); \
    prod = prod + ((YO(23) * YO(13)) * RCS(84)); \
    loss = loss + ((YO(18) * YN(2)) * RCS(85)); \
    prod = prod + (YO(23) * RCT(0, 2)); \
    loss = loss + (YO(13) * RCT(0, 3)); \
    prod = prod + (YO(34) * RCT(0, 4)); \
    loss = loss + (YO(13) * RCT(0, 5)); \
    prod = prod + ((YO(18) * YO(9)) * RCS(147)); \
    loss = loss + (YO(35) * RCS(146)); \
    prod = prod + (YN(3) * (YO(36) * RCS(166))); \
    loss = loss + (YO(16) * RCS(167)); \
    prod = prod + ((YO(37) * YO(10)) * RCS(186)); \
    loss = loss + (YO(36) * RCS(187)); \
    prod = prod + (YN(6) * (YO(37) * RCS(188))); \
    loss = loss + ((YN(4) * YO(22)) * RCS(189)); \
    prod = prod + (YN(1) * (YO(36) * RCS(190))); \
    loss = loss + ((YO(13) * YO(10)) * RCS(191)); \
    prod = prod + ((0.5 * SOUR(2)) * YN(1)); \
    prod = prod + (SOUR(3) * YN(4)); \
    prod = prod + (SOUR(4) * YN(3)); \
    rhs1 = rho * Y0S(0) + dt * WM(8) * (prod + extra); \
    rhs2 = -(dt * WM(8) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(8) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(8) - fnew); \
    UC_UPDATE_TAIL(8); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 10); \
    prod = (YN(8) * (YN(4) * RCT(0, 6))); \
    extra = 0.0; \
    loss = (YN(2) * RCT(0, 7)); \
    prod = prod + (YN(8) * (YN(6) * RCT(0, 8))); \
    loss = loss + (YN(4) * RCT(0, 9)); \
    prod = prod + (YN(8) * (YN(1) * RCT(0, 10))); \
    loss = loss + (YN(3) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 106); \
    TM_LD(0, 1, 104); \
    TM_LD(0, 2, 110); \
    TM_LD(0, 3, 108); \
    TM_LD(0, 4, 114); \
    TM_LD(0, 5, 112); \
    TM_LD(0, 6, 118); \
    TM_LD(0, 7, 116); \
    TM_LD(0, 8, 122); \
    TM_LD(0, 9, 120); \
    TM_LD(0, 10, 126); \
    TM_LD(0, 11, 124); \
    prod = prod + (YN(3) * (YO(10) * RCT(1, 0))); \
    loss = loss + (YN(2) * RCT(1, 1)); \
    prod = prod + (YN(8) * (YO(11) * RCT(1, 2))); \
    loss = loss + (YO(15) * RCT(1, 3)); \
    prod = prod + (YN(1) * (YO(14) * RCT(1, 4))); \
    loss = loss + (YN(0) * RCT(1, 5)); \
    prod = prod + (YN(8) * (YO(10) * RCT(1, 6))); \
    loss = loss + (YO(20) * RCT(1, 7)); \
    prod = prod + (YN(3) * (YO(25) * RCS(24))); \
    loss = loss + (YO(14) * RCS(25)); \
    prod = prod + (YN(1) * (YO(26) * RCS(38))); \
    loss = loss + ((YN(8) * YN(2)) * RCS(39)); \
    prod = prod + (YN(1) * (YO(27) * RCS(46))); \
    loss = loss + (YO(20) * RCS(47)); \
    prod = prod + (YN(8) * (YO(35) * RCS(146))); \
    loss = loss + (YO(18) * RCS(147)); \
    rhs1 = rho * Y0S(1) + dt * WM(9) * (prod + extra); \
    rhs2 = -(dt * WM(9) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(9) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(9) - fnew); \
    UC_UPDATE_TAIL(9); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 11); \
    prod = (YN(8) * (YN(2) * RCT(1, 8))); \
    extra = 0.0; \
    loss = RCT(1, 9); \
    prod = prod + (YN(8) * (YN(0) * RCT(1, 10))); \
    loss = loss + (YN(2) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 128); \
    TM_LD(1, 1, 130); \
    TM_LD(1, 2, 132); \
    TM_LD(1, 3, 134); \
    TM_LD(1, 4, 136); \
    TM_LD(1, 5, 138); \
    TM_LD(1, 6, 140); \
    TM_LD(1, 7, 142); \
    TM_LD(1, 8, 144); \
    TM_LD(1, 9, 146); \
    TM_LD(1, 10, 252); \
    TM_LD(1, 11, 254); \
    prod = prod + (YN(8) * (YN(4) * RCT(0, 0))); \
    loss = loss + (YN(3) * RCT(0, 1)); \
    prod = prod + (YN(9) * (YN(2) * RCT(0, 2))); \
    loss = loss + (YN(3) * RCT(0, 3)); \
    prod = prod + (YN(8) * (YN(5) * RCT(0, 4))); \
    loss = loss + (YN(4) * RCT(0, 5)); \
    prod = prod + (YN(8) * (YN(6) * RCT(0, 6))); \
    loss = loss + (YN(1) * RCT(0, 7)); \
    prod = prod + (YN(8) * (YO(12) * RCT(0, 8))); \
    loss = loss + (YO(13) * RCT(0, 9)); \
    prod = prod + (YO(11) * RCT(0, 10)); \
    loss = loss + (YN(2) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 260); \
    TM_LD(0, 1, 262); \
    TM_LD(0, 2, 340); \
    TM_LD(0, 3, 342); \
    TM_LD(0, 4, 376); \
    TM_LD(0, 5, 378); \
    TM_LD(0, 6, 404); \
    TM_LD(0, 7, 406); \
    TM_LD(0, 8, 124); \
    TM_LD(0, 9, 126); \
    TM_LD(0, 10, 130); \
    TM_LD(0, 11, 128); \
    prod = prod + (YN(2) * (YO(11) * RCT(1, 0))); \
    loss = loss + (YN(0) * RCT(1, 1)); \
    prod = prod + (YN(3) * (YO(11) * RCT(1, 2))); \
    loss = loss + (YN(4) * RCT(1, 3)); \
    prod = prod + (YN(4) * (YO(11) * RCT(1, 4))); \
    loss = loss + (YN(5) * RCT(1, 5)); \
    prod = prod + (YN(1) * (YO(11) * RCT(1, 6))); \
    loss = loss + (YN(6) * RCT(1, 7)); \
    prod = prod + (YN(6) * (YO(11) * RCT(1, 8))); \
    loss = loss + (YN(7) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(20) * RCT(1, 10))); \
    loss = loss + (YN(3) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 134); \
    TM_LD(1, 1, 132); \
    TM_LD(1, 2, 138); \
    TM_LD(1, 3, 136); \
    TM_LD(1, 4, 142); \
    TM_LD(1, 5, 140); \
    TM_LD(1, 6, 146); \
    TM_LD(1, 7, 144); \
    TM_LD(1, 8, 180); \
    TM_LD(1, 9, 182); \
    TM_LD(1, 10, 192); \
    TM_LD(1, 11, 194); \
    prod = prod + (YN(9) * (YO(20) * RCT(0, 0))); \
    loss = loss + (YN(8) * RCT(0, 1)); \
    prod = prod + (YN(3) * (YO(16) * RCT(0, 2))); \
    loss = loss + (YO(13) * RCT(0, 3)); \
    prod = prod + (YN(1) * (YO(22) * RCT(0, 4))); \
    loss = loss + (YO(11) * RCT(0, 5)); \
    prod = prod + (YN(4) * (YO(26) * RCS(32))); \
    loss = loss + ((YN(8) * YN(2)) * RCS(33)); \
    prod = prod + (YN(1) * (YO(27) * RCS(48))); \
    loss = loss + (YN(8) * RCS(49)); \
    prod = prod + (YN(2) * (YO(23) * RCS(74))); \
    loss = loss + (YO(13) * RCS(75)); \
    prod = prod + (YN(3) * (YO(23) * RCS(78))); \
    loss = loss + (YO(11) * RCS(79)); \
    prod = prod + (YN(6) * (YO(23) * RCS(86))); \
    loss = loss + ((YO(11) * YN(4)) * RCS(87)); \
    prod = prod + (YO(31) * RCT(0, 6)); \
    loss = loss + (YO(13) * RCT(0, 7)); \
    prod = prod + (YN(1) * (YO(37) * RCS(176))); \
    loss = loss + (YO(25) * RCS(177)); \
    prod = prod + (YN(8) * (YO(36) * RCS(187))); \
    loss = loss + (YO(37) * RCS(186)); \
    prod = prod + (YN(1) * (YO(36) * RCS(190))); \
    loss = loss + ((YO(13) * YN(8)) * RCS(191)); \
    prod = prod + (YN(3) * (YO(39) * RCS(192))); \
    loss = loss + (YO(18) * RCS(193)); \
    rhs1 = rho * Y0S(0) + dt * WM(10) * (prod + extra); \
    rhs2 = -(dt * WM(10) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(10) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(10) - fnew); \
    UC_UPDATE_TAIL(10); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 12); \
    prod = (YN(10) * (YN(2) * RCT(0, 8))); \
    extra = 0.0; \
    loss = RCT(0, 9); \
    prod = prod + (YN(10) * (YN(0) * RCT(0, 10))); \
    loss = loss + (YN(2) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 216); \
    TM_LD(0, 1, 218); \
    TM_LD(0, 2, 220); \
    TM_LD(0, 3, 222); \
    TM_LD(0, 4, 232); \
    TM_LD(0, 5, 234); \
    TM_LD(0, 6, 256); \
    TM_LD(0, 7, 258); \
    TM_LD(0, 8, 264); \
    TM_LD(0, 9, 266); \
    TM_LD(0, 10, 272); \
    TM_LD(0, 11, 274); \
    prod = prod + (YN(10) * (YN(4) * RCT(1, 0))); \
    loss = loss + (YN(3) * RCT(1, 1)); \
    prod = prod + (YN(10) * (YN(5) * RCT(1, 2))); \
    loss = loss + (YN(4) * RCT(1, 3)); \
    prod = prod + (YN(10) * (YN(6) * RCT(1, 4))); \
    loss = loss + (YN(1) * RCT(1, 5)); \
    prod = prod + (YN(10) * (YN(7) * RCT(1, 6))); \
    loss = loss + (YN(6) * RCT(1, 7)); \
    prod = prod + (YN(3) * (YO(13) * RCT(1, 8))); \
    loss = loss + (YN(2) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(13) * RCT(1, 10))); \
    loss = loss + (YN(4) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 276); \
    TM_LD(1, 1, 278); \
    TM_LD(1, 2, 280); \
    TM_LD(1, 3, 282); \
    TM_LD(1, 4, 284); \
    TM_LD(1, 5, 286); \
    TM_LD(1, 6, 320); \
    TM_LD(1, 7, 322); \
    TM_LD(1, 8, 376); \
    TM_LD(1, 9, 378); \
    TM_LD(1, 10, 384); \
    TM_LD(1, 11, 386); \
    prod = prod + (YN(4) * (YO(15) * RCT(0, 0))); \
    loss = loss + (YN(2) * RCT(0, 1)); \
    prod = prod + (YN(9) * (YO(15) * RCT(0, 2))); \
    loss = loss + (YN(8) * RCT(0, 3)); \
    prod = prod + (YN(4) * (YO(14) * RCT(0, 4))); \
    loss = loss + (YN(2) * RCT(0, 5)); \
    prod = prod + (YN(5) * (YO(20) * RCT(0, 6))); \
    loss = loss + (YN(2) * RCT(0, 7)); \
    prod = prod + (YN(2) * (YO(17) * RCT(0, 8))); \
    loss = loss + (YN(0) * RCT(0, 9)); \
    prod = prod + (YN(4) * (YO(17) * RCT(0, 10))); \
    loss = loss + (YN(5) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 428); \
    TM_LD(0, 1, 430); \
    TM_LD(0, 2, 120); \
    TM_LD(0, 3, 122); \
    TM_LD(0, 4, 150); \
    TM_LD(0, 5, 148); \
    TM_LD(0, 6, 154); \
    TM_LD(0, 7, 152); \
    TM_LD(0, 8, 158); \
    TM_LD(0, 9, 156); \
    TM_LD(0, 10, 162); \
    TM_LD(0, 11, 160); \
    prod = prod + (YN(3) * (YO(17) * RCT(1, 0))); \
    loss = loss + (YN(4) * RCT(1, 1)); \
    prod = prod + (YN(1) * (YO(17) * RCT(1, 2))); \
    loss = loss + (YN(6) * RCT(1, 3)); \
    prod = prod + (YO(17) * RCT(1, 4)); \
    loss = loss + (YN(2) * RCT(1, 5)); \
    prod = prod + (YN(3) * (YO(18) * RCT(1, 6))); \
    loss = loss + (YO(13) * RCT(1, 7)); \
    prod = prod + (YN(1) * (YO(22) * RCT(1, 8))); \
    loss = loss + (YN(10) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(21) * RCS(16))); \
    loss = loss + (YN(8) * RCS(17)); \
    prod = prod + (YN(2) * (YO(28) * RCS(50))); \
    loss = loss + (YN(0) * RCS(51)); \
    prod = prod + (YN(4) * (YO(28) * RCS(54))); \
    loss = loss + (YN(5) * RCS(55)); \
    prod = prod + (YN(1) * (YO(28) * RCS(56))); \
    loss = loss + (YN(6) * RCS(57)); \
    prod = prod + (YO(28) * RCT(1, 10)); \
    loss = loss + (YN(2) * RCT(1, 11)); \
    prod = prod + (YN(3) * (YO(23) * RCS(78))); \
    loss = loss + (YN(10) * RCS(79)); \
    prod = prod + (YN(1) * (YO(23) * RCS(82))); \
    loss = loss + ((YN(8) * YN(4)) * RCS(83)); \
    prod = prod + (YN(6) * (YO(23) * RCS(86))); \
    loss = loss + ((YN(10) * YN(4)) * RCS(87)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 166); \
    TM_LD(1, 1, 164); \
    TM_LD(1, 2, 208); \
    TM_LD(1, 3, 210); \
    TM_LD(1, 4, 300); \
    TM_LD(1, 5, 302); \
    TM_LD(1, 6, 122); \
    TM_LD(1, 7, 120); \
    TM_LD(1, 8, 148); \
    TM_LD(1, 9, 150); \
    TM_LD(1, 10, 152); \
    TM_LD(1, 11, 154); \
    prod = prod + (YO(35) * RCT(0, 0)); \
    loss = loss + (YO(13) * RCT(0, 1)); \
    prod = prod + (YN(6) * (YO(38) * RCS(202))); \
    loss = loss + ((YN(4) * YO(22)) * RCS(203)); \
    rhs1 = rho * Y0S(1) + dt * WM(11) * (prod + extra); \
    rhs2 = -(dt * WM(11) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(11) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(11) - fnew); \
    UC_UPDATE_TAIL(11); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 13); \
    prod = (YN(10) * (YO(13) * RCT(0, 2))); \
    extra = 0.0; \
    loss = (YN(8) * RCT(0, 3)); \
    prod = prod + (YN(0) * (YO(13) * RCT(0, 4))); \
    loss = loss + (YN(2) * RCT(0, 5)); \
    prod = prod + (YN(5) * (YO(13) * RCT(0, 6))); \
    loss = loss + (YN(4) * RCT(0, 7)); \
    prod = prod + (YN(4) * (YO(13) * RCT(0, 8))); \
    loss = loss + (YN(3) * RCT(0, 9)); \
    prod = prod + (YN(6) * (YO(13) * RCT(0, 10))); \
    loss = loss + (YN(1) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 156); \
    TM_LD(0, 1, 158); \
    TM_LD(0, 2, 160); \
    TM_LD(0, 3, 162); \
    TM_LD(0, 4, 164); \
    TM_LD(0, 5, 166); \
    TM_LD(0, 6, 170); \
    TM_LD(0, 7, 168); \
    TM_LD(0, 8, 174); \
    TM_LD(0, 9, 172); \
    TM_LD(0, 10, 178); \
    TM_LD(0, 11, 176); \
    prod = prod + (YN(7) * (YO(13) * RCT(1, 0))); \
    loss = loss + (YN(6) * RCT(1, 1)); \
    prod = prod + (YN(2) * (YO(13) * RCT(1, 2))); \
    loss = loss + RCT(1, 3); \
    prod = prod + ((YO(19) * YO(13)) * RCT(1, 4)); \
    loss = loss + (YO(18) * RCT(1, 5)); \
    prod = prod + ((YO(31) * YO(13)) * RCS(102)); \
    loss = loss + (YO(34) * RCS(103)); \
    prod = prod + ((YO(31) * YO(13)) * RCS(104)); \
    loss = loss + (YO(23) * RCS(105)); \
    prod = prod + ((YO(30) * YO(13)) * RCS(130)); \
    loss = loss + (YO(33) * RCS(131)); \
    prod = prod + ((YO(30) * YO(13)) * RCS(132)); \
    loss = loss + (YO(32) * RCS(133)); \
    prod = prod + ((YO(30) * YO(13)) * RCS(134)); \
    loss = loss + (YO(35) * RCS(135)); \
    prod = prod + ((YO(38) * YO(13)) * RCS(182)); \
    loss = loss + (YO(36) * RCS(183)); \
    prod = prod + ((YO(43) * YO(13)) * RCS(240)); \
    loss = loss + ((YO(21) * YO(22)) * RCS(241)); \
    rhs1 = rho * Y0S(0) + dt * WM(12) * (prod + extra); \
    rhs2 = -(dt * WM(12) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(12) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(12) - fnew); \
    UC_UPDATE_TAIL(12); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 14); \
    prod = (YN(12) * (YN(8) * RCT(1, 6))); \
    extra = (1.0 * (YO(46) * RCS(250))); \
    loss = (YN(10) * RCT(1, 7)); \
    prod = prod + (YN(12) * (YN(2) * RCT(1, 8))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(252)))); \
    loss = loss + (YN(0) * RCT(1, 9)); \
    prod = prod + (YN(12) * (YN(4) * RCT(1, 10))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(253)))); \
    loss = loss + (YN(5) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 182); \
    TM_LD(1, 1, 180); \
    TM_LD(1, 2, 186); \
    TM_LD(1, 3, 184); \
    TM_LD(1, 4, 190); \
    TM_LD(1, 5, 188); \
    TM_LD(1, 6, 194); \
    TM_LD(1, 7, 192); \
    TM_LD(1, 8, 198); \
    TM_LD(1, 9, 196); \
    TM_LD(1, 10, 202); \
    TM_LD(1, 11, 200); \
    prod = prod + (YN(12) * (YN(3) * RCT(0, 0))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(258)))); \
    loss = loss + (YN(4) * RCT(0, 1)); \
    prod = prod + (YN(12) * (YN(1) * RCT(0, 2))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    loss = loss + (YN(6) * RCT(0, 3)); \
    prod = prod + (YN(12) * (YN(6) * RCT(0, 4))); \
    loss = loss + (YN(7) * RCT(0, 5)); \
    prod = prod + (YN(0) * (YO(14) * RCT(0, 6))); \
    loss = loss + (YN(2) * RCT(0, 7)); \
    prod = prod + (YN(0) * (YO(15) * RCT(0, 8))); \
    loss = loss + (YN(2) * RCT(0, 9)); \
    prod = prod + (YN(5) * (YO(15) * RCT(0, 10))); \
    loss = loss + (YN(4) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 206); \
    TM_LD(0, 1, 204); \
    TM_LD(0, 2, 210); \
    TM_LD(0, 3, 208); \
    TM_LD(0, 4, 214); \
    TM_LD(0, 5, 212); \
    TM_LD(0, 6, 302); \
    TM_LD(0, 7, 300); \
    TM_LD(0, 8, 320); \
    TM_LD(0, 9, 322); \
    TM_LD(0, 10, 340); \
    TM_LD(0, 11, 342); \
    prod = prod + (YN(11) * (YN(2) * RCT(1, 0))); \
    loss = loss + (YN(3) * RCT(1, 1)); \
    prod = prod + (YN(2) * (YO(16) * RCT(1, 2))); \
    loss = loss + (YO(14) * RCT(1, 3)); \
    prod = prod + (YN(4) * (YO(17) * RCT(1, 4))); \
    loss = loss + (YN(6) * RCT(1, 5)); \
    prod = prod + (YN(11) * (YN(4) * RCT(1, 6))); \
    loss = loss + (YN(1) * RCT(1, 7)); \
    prod = prod + (YN(3) * (YO(17) * RCT(1, 8))); \
    loss = loss + (YN(1) * RCT(1, 9)); \
    prod = prod + (YN(0) * (YO(16) * RCT(1, 10))); \
    loss = loss + (YO(13) * RCT(1, 11)); \
    prod = prod + (YN(0) * (YO(16) * RCT(1, 10))); \
    loss = loss + (YO(13) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 392); \
    TM_LD(1, 1, 394); \
    TM_LD(1, 2, 400); \
    TM_LD(1, 3, 402); \
    TM_LD(1, 4, 404); \
    TM_LD(1, 5, 406); \
    TM_LD(1, 6, 408); \
    TM_LD(1, 7, 410); \
    TM_LD(1, 8, 412); \
    TM_LD(1, 9, 414); \
    TM_LD(1, 10, 428); \
    TM_LD(1, 11, 430); \
    prod = prod + (YN(2) * (YO(18) * RCT(0, 0))); \
    loss = loss + (YO(13) * RCT(0, 1)); \
    prod = prod + (YN(2) * (YO(18) * RCT(0, 0))); \
    loss = loss + (YO(13) * RCT(0, 1)); \
    prod = prod + (YN(12) * RCT(0, 2)); \
    loss = loss + (YN(2) * RCT(0, 3)); \
    prod = prod + (YO(19) * RCT(0, 4)); \
    loss = loss + (YO(13) * RCT(0, 5)); \
    prod = prod + (YO(19) * RCT(0, 4)); \
    loss = loss + (YO(13) * RCT(0, 5)); \
    prod = prod + (YN(12) * (YO(18) * RCT(0, 6))); \
    loss = loss + (YO(19) * RCT(0, 7)); \
    prod = prod + (YN(3) * (YO(18) * RCT(0, 8))); \
    loss = loss + (YN(11) * RCT(0, 9)); \
    prod = prod + (YN(3) * (YO(16) * RCT(0, 10))); \
    loss = loss + (YN(10) * RCT(0, 11)); \
    prod = prod + (YN(6) * (YO(24) * RCS(8))); \
    loss = loss + ((YN(8) * YN(7)) * RCS(9)); \
    prod = prod + (YN(2) * (YO(25) * RCS(22))); \
    loss = loss + (YN(8) * RCS(23)); \
    prod = prod + (YN(8) * (YO(18) * RCS(29))); \
    loss = loss + (YO(25) * RCS(28)); \
    prod = prod + (YN(2) * (YO(28) * RCS(52))); \
    loss = loss + (YN(4) * RCS(53)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 446); \
    TM_LD(0, 1, 444); \
    TM_LD(0, 2, 454); \
    TM_LD(0, 3, 452); \
    TM_LD(0, 4, 456); \
    TM_LD(0, 5, 458); \
    TM_LD(0, 6, 468); \
    TM_LD(0, 7, 470); \
    TM_LD(0, 8, 486); \
    TM_LD(0, 9, 484); \
    TM_LD(0, 10, 508); \
    TM_LD(0, 11, 510); \
    prod = prod + (YO(29) * RCT(1, 0)); \
    loss = loss + (YN(4) * RCT(1, 1)); \
    prod = prod + (YN(2) * (YO(23) * RCS(74))); \
    loss = loss + (YN(10) * RCS(75)); \
    prod = prod + (YN(8) * ((YO(18) * YN(2)) * RCS(85))); \
    loss = loss + (YO(23) * RCS(84)); \
    prod = prod + (YO(23) * RCT(1, 2)); \
    loss = loss + (YN(8) * RCT(1, 3)); \
    prod = prod + (YO(31) * RCT(1, 4)); \
    loss = loss + (YN(10) * RCT(1, 5)); \
    prod = prod + (YO(34) * RCT(1, 6)); \
    loss = loss + (YN(8) * RCT(1, 7)); \
    prod = prod + (YN(12) * (YO(34) * RCS(103))); \
    loss = loss + (YO(31) * RCS(102)); \
    prod = prod + (YN(12) * (YO(23) * RCS(105))); \
    loss = loss + (YO(31) * RCS(104)); \
    prod = prod + (YO(30) * RCT(1, 8)); \
    loss = loss + (YO(28) * RCT(1, 9)); \
    prod = prod + (YN(12) * (YO(33) * RCS(131))); \
    loss = loss + (YO(30) * RCS(130)); \
    prod = prod + (YN(12) * (YO(32) * RCS(133))); \
    loss = loss + (YO(30) * RCS(132)); \
    prod = prod + (YN(12) * (YO(35) * RCS(135))); \
    loss = loss + (YO(30) * RCS(134)); \
    prod = prod + (YO(35) * RCT(1, 10)); \
    loss = loss + (YN(11) * RCT(1, 11)); \
    prod = prod + (YN(2) * (YO(35) * RCS(148))); \
    loss = loss + (YO(28) * RCS(149)); \
    prod = prod + (YN(2) * (YO(32) * RCS(160))); \
    loss = loss + (YO(28) * RCS(161)); \
    prod = prod + (YN(2) * (YO(36) * RCS(169))); \
    loss = loss + (YO(21) * RCS(168)); \
    prod = prod + (YN(3) * (YO(36) * RCS(170))); \
    loss = loss + (YO(26) * RCS(171)); \
    prod = prod + (YN(12) * (YO(36) * RCS(183))); \
    loss = loss + (YO(38) * RCS(182)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 168); \
    TM_LD(1, 1, 170); \
    TM_LD(1, 2, 186); \
    TM_LD(1, 3, 184); \
    TM_LD(1, 4, 224); \
    TM_LD(1, 5, 226); \
    TM_LD(1, 6, 230); \
    TM_LD(1, 7, 228); \
    TM_LD(1, 8, 234); \
    TM_LD(1, 9, 232); \
    TM_LD(1, 10, 238); \
    TM_LD(1, 11, 236); \
    prod = prod + (YO(38) * RCT(0, 0)); \
    loss = loss + (YO(21) * RCT(0, 1)); \
    prod = prod + (YN(1) * (YO(36) * RCS(190))); \
    loss = loss + ((YN(10) * YN(8)) * RCS(191)); \
    prod = prod + (YN(3) * (YO(39) * RCS(196))); \
    loss = loss + ((YO(25) * YN(2)) * RCS(197)); \
    prod = prod + (YO(39) * RCT(0, 2)); \
    loss = loss + (YO(22) * RCT(0, 3)); \
    prod = prod + (YN(2) * (YO(39) * RCS(204))); \
    loss = loss + (YO(16) * RCS(205)); \
    prod = prod + (YN(2) * (YO(38) * RCS(207))); \
    loss = loss + (YO(22) * RCS(206)); \
    prod = prod + (YO(40) * RCT(0, 4)); \
    loss = loss + (YO(18) * RCT(0, 5)); \
    prod = prod + (YO(42) * RCT(0, 6)); \
    loss = loss + (YO(16) * RCT(0, 7)); \
    prod = prod + (YN(12) * ((YO(21) * YO(22)) * RCS(241))); \
    loss = loss + (YO(43) * RCS(240)); \
    prod = prod + (YO(43) * RCT(0, 8)); \
    loss = loss + (YO(37) * RCT(0, 9)); \
    prod = prod + (YN(2) * (YO(48) * RCS(265))); \
    loss = loss + ((YO(16) * YO(16)) * RCS(266)); \
    prod = prod + (YN(2) * (YO(48) * RCS(271))); \
    loss = loss + ((YN(0) * YO(43)) * RCS(272)); \
    prod = prod + (YO(47) * RCT(0, 10)); \
    loss = loss + (YO(38) * RCT(0, 11)); \
    prod = prod + (YN(2) * (YO(47) * RCS(275))); \
    loss = loss + (YO(39) * RCS(276)); \
    rhs1 = rho * Y0S(1) + dt * WM(13) * (prod + extra); \
    rhs2 = -(dt * WM(13) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(13) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(13) - fnew); \
    UC_UPDATE_TAIL(13); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 15); \
    TM_WAIT(1); \
    TM_LD(0, 0, 242); \
    TM_LD(0, 1, 240); \
    TM_LD(0, 2, 246); \
    TM_LD(0, 3, 244); \
    TM_LD(0, 4, 172); \
    TM_LD(0, 5, 174); \
    TM_LD(0, 6, 176); \
    TM_LD(0, 7, 178); \
    TM_LD(0, 8, 218); \
    TM_LD(0, 9, 216); \
    TM_LD(0, 10, 222); \
    TM_LD(0, 11, 220); \
    prod = (YN(13) * (YN(2) * RCT(1, 0))); \
    extra = 0.0; \
    loss = (YN(0) * RCT(1, 1)); \
    prod = prod + (YN(2) * (YO(16) * RCT(1, 2))); \
    loss = loss + (YN(13) * RCT(1, 3)); \
    prod = prod + (YO(15) * RCT(1, 4)); \
    loss = loss + RCT(1, 5); \
    prod = prod + (YN(0) * (YO(20) * RCT(1, 6))); \
    loss = loss + (YN(2) * RCT(1, 7)); \
    prod = prod + (YN(11) * (YN(2) * RCT(1, 8))); \
    loss = loss + (YN(4) * RCT(1, 9)); \
    prod = prod + (YN(5) * (YO(20) * RCT(1, 10))); \
    loss = loss + (YN(4) * RCT(1, 11)); \
    prod = prod + (YN(8) * ((YN(2) * YN(2)) * RCS(3))); \
    loss = loss + (YN(3) * RCS(2)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 226); \
    TM_LD(1, 1, 224); \
    TM_LD(1, 2, 268); \
    TM_LD(1, 3, 270); \
    TM_LD(1, 4, 184); \
    TM_LD(1, 5, 186); \
    TM_LD(1, 6, 200); \
    TM_LD(1, 7, 202); \
    TM_LD(1, 8, 312); \
    TM_LD(1, 9, 314); \
    TM_LD(1, 10, 316); \
    TM_LD(1, 11, 318); \
    prod = prod + (YN(8) * (YN(0) * RCT(0, 0))); \
    loss = loss + (YN(3) * RCT(0, 1)); \
    prod = prod + (YN(9) * (YN(0) * RCT(0, 2))); \
    loss = loss + (YN(1) * RCT(0, 3)); \
    prod = prod + (YN(8) * ((YN(4) * YN(2)) * RCS(5))); \
    loss = loss + (YN(1) * RCS(4)); \
    prod = prod + (YN(2) * ((YO(21) * YOS(0)) * RCS(7))); \
    loss = loss + (YO(14) * RCS(6)); \
    prod = prod + (YN(2) * ((YO(21) * YOS(0)) * RCS(7))); \
    loss = loss + (YO(14) * RCS(6)); \
    prod = prod + (YN(3) * (YO(21) * RCS(14))); \
    loss = loss + (YN(8) * RCS(15)); \
    prod = prod + (YN(3) * (YO(25) * RCS(24))); \
    loss = loss + (YN(9) * RCS(25)); \
    rhs1 = rho * Y0S(0) + dt * WM(14) * (prod + extra); \
    rhs2 = -(dt * WM(14) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(14) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(14) - fnew); \
    UC_UPDATE_TAIL(14); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 16); \
    prod = (YN(13) * (YN(2) * RCT(0, 4))); \
    extra = 0.0; \
    loss = (YN(0) * RCT(0, 5)); \
    prod = prod + (YN(13) * (YN(4) * RCT(0, 6))); \
    loss = loss + (YN(5) * RCT(0, 7)); \
    prod = prod + (YN(11) * (YN(2) * RCT(0, 8))); \
    loss = loss + (YN(4) * RCT(0, 9)); \
    prod = prod + (YN(8) * ((YN(4) * YN(2)) * RCS(1))); \
    loss = loss + (YN(1) * RCS(0)); \
    prod = prod + (YN(11) * (YN(8) * RCT(0, 10))); \
    loss = loss + (YN(9) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 324); \
    TM_LD(0, 1, 326); \
    TM_LD(0, 2, 328); \
    TM_LD(0, 3, 330); \
    TM_LD(0, 4, 334); \
    TM_LD(0, 5, 332); \
    TM_LD(0, 6, 338); \
    TM_LD(0, 7, 336); \
    TM_LD(0, 8, 342); \
    TM_LD(0, 9, 340); \
    TM_LD(0, 10, 346); \
    TM_LD(0, 11, 344); \
    prod = prod + (YN(14) * RCT(1, 0)); \
    loss = loss + RCT(1, 1); \
    prod = prod + (YN(2) * (YO(17) * RCT(1, 2))); \
    loss = loss + (YN(5) * RCT(1, 3)); \
    prod = prod + (YN(2) * (YO(26) * RCS(30))); \
    loss = loss + (YN(8) * RCS(31)); \
    rhs1 = rho * Y0S(1) + dt * WM(15) * (prod + extra); \
    rhs2 = -(dt * WM(15) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(15) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(15) - fnew); \
    UC_UPDATE_TAIL(15); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 17); \
    prod = (YN(14) * (YN(13) * RCT(1, 4))); \
    extra = (1.0 * (YO(46) * RCS(250))); \
    loss = (YN(2) * RCT(1, 5)); \
    prod = prod + (YN(13) * (YOS(3) * RCT(1, 6))); \
    extra = extra + (1.0 * (YO(46) * RCS(250))); \
    loss = loss + (YN(0) * RCT(1, 7)); \
    prod = prod + (YN(2) * (YO(18) * RCT(1, 8))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(251)))); \
    loss = loss + (YN(0) * RCT(1, 9)); \
    prod = prod + (YN(3) * (YO(18) * RCT(1, 10))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(252)))); \
    loss = loss + (YN(4) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 350); \
    TM_LD(1, 1, 348); \
    TM_LD(1, 2, 354); \
    TM_LD(1, 3, 352); \
    TM_LD(1, 4, 358); \
    TM_LD(1, 5, 356); \
    TM_LD(1, 6, 362); \
    TM_LD(1, 7, 360); \
    TM_LD(1, 8, 366); \
    TM_LD(1, 9, 364); \
    TM_LD(1, 10, 416); \
    TM_LD(1, 11, 418); \
    prod = prod + (YN(1) * (YO(18) * RCT(0, 0))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(253)))); \
    loss = loss + (YN(6) * RCT(0, 1)); \
    prod = prod + (YO(18) * RCT(0, 2)); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(253)))); \
    loss = loss + (YN(2) * RCT(0, 3)); \
    prod = prod + (YN(0) * (YO(22) * RCT(0, 4))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(253)))); \
    loss = loss + (YN(2) * RCT(0, 5)); \
    prod = prod + (YN(5) * (YO(22) * RCT(0, 6))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(258)))); \
    loss = loss + (YN(4) * RCT(0, 7)); \
    prod = prod + (YN(13) * (YN(10) * RCT(0, 8))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(259)))); \
    loss = loss + (YN(3) * RCT(0, 9)); \
    prod = prod + (YN(2) * (YO(23) * RCT(0, 10))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    loss = loss + (YN(3) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 422); \
    TM_LD(0, 1, 420); \
    TM_LD(0, 2, 468); \
    TM_LD(0, 3, 470); \
    TM_LD(0, 4, 492); \
    TM_LD(0, 5, 494); \
    TM_LD(0, 6, 504); \
    TM_LD(0, 7, 506); \
    TM_LD(0, 8, 188); \
    TM_LD(0, 9, 190); \
    TM_LD(0, 10, 196); \
    TM_LD(0, 11, 198); \
    prod = prod + ((YO(22) * YO(18)) * RCT(1, 0)); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    loss = loss + (YO(16) * RCT(1, 1)); \
    prod = prod + ((YO(22) * YO(18)) * RCT(1, 0)); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    loss = loss + (YO(16) * RCT(1, 1)); \
    prod = prod + (YN(6) * (YO(22) * RCT(1, 2))); \
    loss = loss + (YN(1) * RCT(1, 3)); \
    prod = prod + (YN(4) * (YO(24) * RCT(1, 4))); \
    loss = loss + (YN(6) * RCT(1, 5)); \
    prod = prod + (YN(2) * (YO(22) * RCT(1, 6))); \
    loss = loss + RCT(1, 7); \
    prod = prod + (YN(0) * (YO(21) * RCT(1, 8))); \
    loss = loss + RCT(1, 9); \
    prod = prod + (YO(30) * RCT(1, 10)); \
    loss = loss + (YN(5) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 266); \
    TM_LD(1, 1, 264); \
    TM_LD(1, 2, 270); \
    TM_LD(1, 3, 268); \
    TM_LD(1, 4, 274); \
    TM_LD(1, 5, 272); \
    TM_LD(1, 6, 278); \
    TM_LD(1, 7, 276); \
    TM_LD(1, 8, 282); \
    TM_LD(1, 9, 280); \
    TM_LD(1, 10, 286); \
    TM_LD(1, 11, 284); \
    prod = prod + (YO(33) * RCT(0, 0)); \
    loss = loss + (YN(4) * RCT(0, 1)); \
    prod = prod + (YN(2) * (YO(35) * RCS(150))); \
    loss = loss + (YN(5) * RCS(151)); \
    prod = prod + (YN(2) * (YO(32) * RCS(158))); \
    loss = loss + (YN(5) * RCS(159)); \
    prod = prod + (YN(3) * (YO(36) * RCS(166))); \
    loss = loss + (YN(8) * RCS(167)); \
    prod = prod + (YN(2) * (YO(39) * RCS(204))); \
    loss = loss + (YN(13) * RCS(205)); \
    prod = prod + (YO(42) * RCT(0, 2)); \
    loss = loss + (YN(13) * RCT(0, 3)); \
    prod = prod + (YN(2) * (YO(43) * RCS(234))); \
    loss = loss + (YO(22) * RCS(235)); \
    prod = prod + (YO(45) * RCT(0, 4)); \
    loss = loss + (YO(36) * RCT(0, 5)); \
    prod = prod + (YO(48) * RCT(0, 6)); \
    loss = loss + (YO(39) * RCT(0, 7)); \
    prod = prod + (YN(2) * (YO(48) * RCS(265))); \
    loss = loss + ((YO(16) * YN(13)) * RCS(266)); \
    prod = prod + (YN(2) * (YO(48) * RCS(265))); \
    loss = loss + ((YO(16) * YN(13)) * RCS(266)); \
    prod = prod + (YN(2) * (YO(48) * RCS(269))); \
    loss = loss + ((YN(0) * YO(38)) * RCS(270)); \
    prod = prod + (YN(2) * (YO(47) * RCS(273))); \
    loss = loss + (YO(18) * RCS(274)); \
    prod = prod + (YN(2) * (YO(47) * RCS(277))); \
    loss = loss + ((YN(0) * YO(22)) * RCS(278)); \
    rhs1 = rho * Y0S(0) + dt * WM(16) * (prod + extra); \
    rhs2 = -(dt * WM(16) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(16) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(16) - fnew); \
    UC_UPDATE_TAIL(16); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 18); \
    prod = (YN(13) * (YN(6) * RCT(0, 8))); \
    extra = 0.0; \
    loss = (YN(4) * RCT(0, 9)); \
    prod = prod + (YN(13) * (YN(1) * RCT(0, 10))); \
    loss = loss + (YN(3) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 390); \
    TM_LD(0, 1, 388); \
    TM_LD(0, 2, 204); \
    TM_LD(0, 3, 206); \
    TM_LD(0, 4, 288); \
    TM_LD(0, 5, 290); \
    TM_LD(0, 6, 292); \
    TM_LD(0, 7, 294); \
    TM_LD(0, 8, 296); \
    TM_LD(0, 9, 298); \
    TM_LD(0, 10, 300); \
    TM_LD(0, 11, 302); \
    prod = prod + (YN(11) * (YN(0) * RCT(1, 0))); \
    loss = loss + (YN(2) * RCT(1, 1)); \
    prod = prod + (YN(15) * (YN(5) * RCT(1, 2))); \
    loss = loss + (YN(2) * RCT(1, 3)); \
    prod = prod + (YN(11) * (YN(5) * RCT(1, 4))); \
    loss = loss + (YN(4) * RCT(1, 5)); \
    prod = prod + (YN(11) * (YN(4) * RCT(1, 6))); \
    loss = loss + (YN(3) * RCT(1, 7)); \
    prod = prod + (YN(11) * (YN(6) * RCT(1, 8))); \
    loss = loss + (YN(1) * RCT(1, 9)); \
    prod = prod + (YN(11) * (YN(2) * RCT(1, 10))); \
    loss = loss + RCT(1, 11); \
    TM_WAIT(0); \
    TM_LD(1, 0, 304); \
    TM_LD(1, 1, 306); \
    TM_LD(1, 2, 308); \
    TM_LD(1, 3, 310); \
    TM_LD(1, 4, 314); \
    TM_LD(1, 5, 312); \
    TM_LD(1, 6, 318); \
    TM_LD(1, 7, 316); \
    TM_LD(1, 8, 322); \
    TM_LD(1, 9, 320); \
    TM_LD(1, 10, 326); \
    TM_LD(1, 11, 324); \
    prod = prod + (YO(28) * RCT(0, 0)); \
    loss = loss + RCT(0, 1); \
    prod = prod + (YN(4) * (YO(29) * RCS(62))); \
    loss = loss + (YN(5) * RCS(63)); \
    prod = prod + (YN(2) * (YO(29) * RCS(66))); \
    loss = loss + (YN(0) * RCS(67)); \
    rhs1 = rho * Y0S(1) + dt * WM(17) * (prod + extra); \
    rhs2 = -(dt * WM(17) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(17) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(17) - fnew); \
    UC_UPDATE_TAIL(17); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 19); \
    prod = (YN(13) * (YOS(3) * RCT(0, 2))); \
    extra = (1.0 * (YO(46) * RCS(250))); \
    loss = (YN(2) * RCT(0, 3)); \
    prod = prod + (YN(2) * (YO(19) * RCT(0, 4))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(251)))); \
    loss = loss + (YN(0) * RCT(0, 5)); \
    prod = prod + (YN(3) * (YO(19) * RCT(0, 6))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(259)))); \
    loss = loss + (YN(4) * RCT(0, 7)); \
    prod = prod + (YN(4) * (YO(19) * RCT(0, 8))); \
    loss = loss + (YN(5) * RCT(0, 9)); \
    prod = prod + (YN(13) * (YO(19) * RCT(0, 10))); \
    loss = loss + (YN(12) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 330); \
    TM_LD(0, 1, 328); \
    TM_LD(0, 2, 348); \
    TM_LD(0, 3, 350); \
    TM_LD(0, 4, 456); \
    TM_LD(0, 5, 458); \
    TM_LD(0, 6, 500); \
    TM_LD(0, 7, 502); \
    TM_LD(0, 8, 212); \
    TM_LD(0, 9, 214); \
    TM_LD(0, 10, 290); \
    TM_LD(0, 11, 288); \
    prod = prod + (YO(19) * RCT(1, 0)); \
    loss = loss + (YN(2) * RCT(1, 1)); \
    prod = prod + (YN(6) * (YO(19) * RCT(1, 2))); \
    loss = loss + (YN(7) * RCT(1, 3)); \
    prod = prod + (YN(16) * (YN(0) * RCT(1, 4))); \
    loss = loss + (YN(2) * RCT(1, 5)); \
    prod = prod + (YN(16) * (YN(4) * RCT(1, 6))); \
    loss = loss + (YN(3) * RCT(1, 7)); \
    prod = prod + (YN(13) * (YN(11) * RCT(1, 8))); \
    loss = loss + (YN(3) * RCT(1, 9)); \
    prod = prod + (YN(16) * (YN(6) * RCT(1, 10))); \
    loss = loss + (YN(1) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 294); \
    TM_LD(1, 1, 292); \
    TM_LD(1, 2, 298); \
    TM_LD(1, 3, 296); \
    TM_LD(1, 4, 302); \
    TM_LD(1, 5, 300); \
    TM_LD(1, 6, 306); \
    TM_LD(1, 7, 304); \
    TM_LD(1, 8, 310); \
    TM_LD(1, 9, 308); \
    TM_LD(1, 10, 228); \
    TM_LD(1, 11, 230); \
    prod = prod + (YN(16) * (YN(2) * RCT(0, 0))); \
    loss = loss + RCT(0, 1); \
    prod = prod + (YN(16) * (YOS(4) * RCT(0, 2))); \
    loss = loss + (YO(22) * RCT(0, 3)); \
    prod = prod + (YN(13) * (YO(25) * RCS(28))); \
    loss = loss + (YN(8) * RCS(29)); \
    prod = prod + (YN(13) * (YO(23) * RCS(84))); \
    loss = loss + ((YN(8) * YN(2)) * RCS(85)); \
    prod = prod + (YN(4) * (YO(35) * RCS(143))); \
    loss = loss + (YN(6) * RCS(142)); \
    prod = prod + (YN(8) * (YO(35) * RCS(146))); \
    loss = loss + (YN(9) * RCS(147)); \
    prod = prod + (YN(3) * (YO(39) * RCS(192))); \
    loss = loss + (YN(10) * RCS(193)); \
    prod = prod + (YO(40) * RCT(0, 4)); \
    loss = loss + (YN(13) * RCT(0, 5)); \
    prod = prod + (YN(2) * (YO(46) * RCS(254))); \
    loss = loss + ((YN(0) * YO(48)) * RCS(255)); \
    prod = prod + (YN(4) * (YO(46) * RCS(256))); \
    loss = loss + ((YN(5) * YO(48)) * RCS(257)); \
    prod = prod + (YO(48) * RCT(0, 6)); \
    loss = loss + (YO(38) * RCT(0, 7)); \
    prod = prod + (YN(2) * (YO(48) * RCS(267))); \
    loss = loss + (YO(39) * RCS(268)); \
    prod = prod + (YN(2) * (YO(47) * RCS(273))); \
    loss = loss + (YN(16) * RCS(274)); \
    rhs1 = rho * Y0S(0) + dt * WM(18) * (prod + extra); \
    rhs2 = -(dt * WM(18) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(18) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(18) - fnew); \
    UC_UPDATE_TAIL(18); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 20); \
    prod = (YN(13) * (YOS(3) * RCT(0, 8))); \
    extra = 0.0; \
    loss = RCT(0, 9); \
    prod = prod + (YN(18) * (YN(0) * RCT(0, 10))); \
    loss = loss + (YN(2) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 236); \
    TM_LD(0, 1, 238); \
    TM_LD(0, 2, 250); \
    TM_LD(0, 3, 248); \
    TM_LD(0, 4, 254); \
    TM_LD(0, 5, 252); \
    TM_LD(0, 6, 258); \
    TM_LD(0, 7, 256); \
    TM_LD(0, 8, 262); \
    TM_LD(0, 9, 260); \
    TM_LD(0, 10, 364); \
    TM_LD(0, 11, 366); \
    prod = prod + (YN(18) * (YN(4) * RCT(1, 0))); \
    loss = loss + (YN(3) * RCT(1, 1)); \
    prod = prod + (YN(18) * (YN(5) * RCT(1, 2))); \
    loss = loss + (YN(4) * RCT(1, 3)); \
    prod = prod + (YN(18) * (YN(12) * RCT(1, 4))); \
    loss = loss + (YN(13) * RCT(1, 5)); \
    prod = prod + (YN(18) * (YN(2) * RCT(1, 6))); \
    loss = loss + RCT(1, 7); \
    prod = prod + (YN(18) * (YN(7) * RCT(1, 8))); \
    loss = loss + (YN(6) * RCT(1, 9)); \
    rhs1 = rho * Y0S(1) + dt * WM(19) * (prod + extra); \
    rhs2 = -(dt * WM(19) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(19) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(19) - fnew); \
    UC_UPDATE_TAIL(19); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 21); \
    prod = (YN(14) * (YN(2) * RCT(1, 10))); \
    extra = 0.0; \
    loss = (YN(0) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 368); \
    TM_LD(1, 1, 370); \
    TM_LD(1, 2, 372); \
    TM_LD(1, 3, 374); \
    TM_LD(1, 4, 446); \
    TM_LD(1, 5, 444); \
    TM_LD(1, 6, 488); \
    TM_LD(1, 7, 490); \
    TM_LD(1, 8, 332); \
    TM_LD(1, 9, 334); \
    TM_LD(1, 10, 336); \
    TM_LD(1, 11, 338); \
    prod = prod + (YN(14) * (YN(4) * RCT(0, 0))); \
    loss = loss + (YN(5) * RCT(0, 1)); \
    prod = prod + (YN(8) * (YN(2) * RCT(0, 2))); \
    loss = loss + (YN(3) * RCT(0, 3)); \
    prod = prod + (YN(10) * (YN(3) * RCT(0, 4))); \
    loss = loss + (YN(1) * RCT(0, 5)); \
    prod = prod + (YN(11) * (YN(2) * RCT(0, 6))); \
    loss = loss + (YN(5) * RCT(0, 7)); \
    prod = prod + (YN(10) * (YN(8) * RCT(0, 8))); \
    loss = loss + (YN(9) * RCT(0, 9)); \
    prod = prod + (YN(3) * (YO(27) * RCS(42))); \
    loss = loss + (YN(8) * RCS(43)); \
    prod = prod + (YN(1) * (YO(27) * RCS(46))); \
    loss = loss + (YN(9) * RCS(47)); \
    rhs1 = rho * Y0S(0) + dt * WM(20) * (prod + extra); \
    rhs2 = -(dt * WM(20) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(20) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(20) - fnew); \
    UC_UPDATE_TAIL(20); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 22); \
    prod = (YN(14) * (YOS(5) * RCS(6))); \
    extra = 0.0; \
    loss = ((YN(2) * YN(2)) * RCS(7)); \
    prod = prod + (YN(16) * RCT(0, 10)); \
    loss = loss + (YN(0) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 348); \
    TM_LD(0, 1, 350); \
    TM_LD(0, 2, 352); \
    TM_LD(0, 3, 354); \
    TM_LD(0, 4, 360); \
    TM_LD(0, 5, 362); \
    TM_LD(0, 6, 370); \
    TM_LD(0, 7, 368); \
    TM_LD(0, 8, 374); \
    TM_LD(0, 9, 372); \
    TM_LD(0, 10, 378); \
    TM_LD(0, 11, 376); \
    prod = prod + (YN(2) * (YO(22) * RCT(1, 0))); \
    loss = loss + (YN(0) * RCT(1, 1)); \
    prod = prod + (YO(22) * RCT(1, 2)); \
    loss = loss + (YN(2) * RCT(1, 3)); \
    prod = prod + (YN(1) * (YO(22) * RCS(10))); \
    loss = loss + (YN(6) * RCS(11)); \
    prod = prod + (YN(2) * (YO(26) * RCS(13))); \
    loss = loss + (YN(3) * RCS(12)); \
    prod = prod + (YN(14) * (YN(8) * RCS(15))); \
    loss = loss + (YN(3) * RCS(14)); \
    prod = prod + (YN(11) * (YN(8) * RCS(17))); \
    loss = loss + (YN(1) * RCS(16)); \
    prod = prod + (YN(2) * (YO(25) * RCS(19))); \
    loss = loss + (YN(4) * RCS(18)); \
    prod = prod + (YN(5) * (YO(27) * RCS(21))); \
    loss = loss + (YN(4) * RCS(20)); \
    prod = prod + (YN(2) * (YO(36) * RCS(169))); \
    loss = loss + (YN(13) * RCS(168)); \
    prod = prod + (YO(38) * RCT(1, 4)); \
    loss = loss + (YN(13) * RCT(1, 5)); \
    prod = prod + (YO(43) * RCS(232)); \
    loss = loss + ((YO(22) * YN(2)) * RCS(233)); \
    prod = prod + (YN(2) * (YO(43) * RCS(236))); \
    loss = loss + ((YN(0) * YO(22)) * RCS(237)); \
    prod = prod + (YN(13) * (YO(43) * RCS(240))); \
    loss = loss + ((YN(12) * YO(22)) * RCS(241)); \
    prod = prod + (YO(45) * RCT(1, 6)); \
    loss = loss + (YO(39) * RCT(1, 7)); \
    prod = prod + (YN(1) * (YO(45) * RCS(242))); \
    loss = loss + ((YO(38) * YN(6)) * RCS(243)); \
    prod = prod + (YN(6) * (YO(45) * RCS(246))); \
    loss = loss + ((YO(38) * YN(7)) * RCS(247)); \
    loss = loss + SOUR(0); \
    rhs1 = rho * Y0S(1) + dt * WM(21) * (prod + extra); \
    rhs2 = -(dt * WM(21) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(21) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(21) - fnew); \
    UC_UPDATE_TAIL(21); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 23); \
    prod = (YN(16) * (YN(2) * RCT(1, 8))); \
    extra = 0.0; \
    loss = (YN(0) * RCT(1, 9)); \
    prod = prod + (YN(16) * (YN(4) * RCT(1, 10))); \
    loss = loss + (YN(5) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 382); \
    TM_LD(1, 1, 380); \
    TM_LD(1, 2, 454); \
    TM_LD(1, 3, 452); \
    TM_LD(1, 4, 476); \
    TM_LD(1, 5, 478); \
    TM_LD(1, 6, 482); \
    TM_LD(1, 7, 480); \
    TM_LD(1, 8, 496); \
    TM_LD(1, 9, 498); \
    TM_LD(1, 10, 344); \
    TM_LD(1, 11, 346); \
    prod = prod + (YN(16) * (YOS(4) * RCT(0, 0))); \
    loss = loss + (YN(18) * RCT(0, 1)); \
    prod = prod + (YN(16) * (YN(1) * RCT(0, 2))); \
    loss = loss + (YN(6) * RCT(0, 3)); \
    prod = prod + (YN(16) * RCT(0, 4)); \
    loss = loss + (YN(2) * RCT(0, 5)); \
    prod = prod + (YN(21) * (YN(0) * RCT(0, 6))); \
    loss = loss + (YN(2) * RCT(0, 7)); \
    prod = prod + (YN(21) * (YN(2) * RCT(0, 8))); \
    loss = loss + RCT(0, 9); \
    prod = prod + (YN(11) * (YN(10) * RCT(0, 10))); \
    loss = loss + (YN(1) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 398); \
    TM_LD(0, 1, 396); \
    TM_LD(0, 2, 402); \
    TM_LD(0, 3, 400); \
    TM_LD(0, 4, 356); \
    TM_LD(0, 5, 358); \
    TM_LD(0, 6, 386); \
    TM_LD(0, 7, 384); \
    TM_LD(0, 8, 388); \
    TM_LD(0, 9, 390); \
    TM_LD(0, 10, 412); \
    TM_LD(0, 11, 414); \
    prod = prod + (YN(3) * (YO(23) * RCT(1, 0))); \
    loss = loss + (YN(1) * RCT(1, 1)); \
    prod = prod + (YN(21) * (YN(6) * RCS(11))); \
    loss = loss + (YN(1) * RCS(10)); \
    prod = prod + (YN(6) * (YO(37) * RCS(188))); \
    loss = loss + ((YN(4) * YN(8)) * RCS(189)); \
    prod = prod + (YN(6) * (YO(38) * RCS(202))); \
    loss = loss + ((YN(4) * YN(11)) * RCS(203)); \
    prod = prod + (YO(39) * RCT(1, 2)); \
    loss = loss + (YN(13) * RCT(1, 3)); \
    prod = prod + (YN(2) * (YO(38) * RCS(207))); \
    loss = loss + (YN(13) * RCS(206)); \
    prod = prod + (YO(43) * RCS(232)); \
    loss = loss + ((YN(21) * YN(2)) * RCS(233)); \
    prod = prod + (YO(43) * RCT(1, 4)); \
    loss = loss + (YO(22) * RCT(1, 5)); \
    prod = prod + (YO(43) * RCT(1, 4)); \
    loss = loss + (YO(22) * RCT(1, 5)); \
    prod = prod + (YO(43) * RCT(1, 6)); \
    loss = loss + (YO(22) * RCT(1, 7)); \
    prod = prod + (YO(43) * RCT(1, 6)); \
    loss = loss + (YO(22) * RCT(1, 7)); \
    prod = prod + (YN(2) * (YO(43) * RCS(234))); \
    loss = loss + (YN(16) * RCS(235)); \
    prod = prod + (YN(2) * (YO(43) * RCS(236))); \
    loss = loss + ((YN(0) * YN(21)) * RCS(237)); \
    prod = prod + (YN(13) * (YO(43) * RCS(240))); \
    loss = loss + ((YN(12) * YN(21)) * RCS(241)); \
    prod = prod + (YO(45) * RCT(1, 8)); \
    loss = loss + (YO(38) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(45) * RCS(244))); \
    loss = loss + ((YO(36) * YN(6)) * RCS(245)); \
    prod = prod + (YN(6) * (YO(45) * RCS(248))); \
    loss = loss + ((YO(36) * YN(7)) * RCS(249)); \
    prod = prod + (YN(4) * (YO(48) * RCS(261))); \
    loss = loss + ((YN(5) * YO(39)) * RCS(262)); \
    prod = prod + (YN(2) * (YO(48) * RCS(263))); \
    loss = loss + ((YN(0) * YO(39)) * RCS(264)); \
    prod = prod + (YN(2) * (YO(47) * RCS(277))); \
    loss = loss + ((YN(0) * YN(16)) * RCS(278)); \
    rhs1 = rho * Y0S(0) + dt * WM(22) * (prod + extra); \
    rhs2 = -(dt * WM(22) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(22) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(22) - fnew); \
    UC_UPDATE_TAIL(22); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 24); \
    prod = (YN(16) * (YN(3) * RCT(1, 10))); \
    extra = 0.0; \
    loss = (YN(2) * RCT(1, 11)); \
    prod = prod + (YN(22) * (YN(1) * RCT(1, 1))); \
    loss = loss + (YN(3) * RCT(1, 0)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 394); \
    TM_LD(1, 1, 392); \
    TM_LD(1, 2, 414); \
    TM_LD(1, 3, 412); \
    TM_LD(1, 4, 418); \
    TM_LD(1, 5, 416); \
    TM_LD(1, 6, 406); \
    TM_LD(1, 7, 404); \
    TM_LD(1, 8, 424); \
    TM_LD(1, 9, 426); \
    TM_LD(1, 10, 432); \
    TM_LD(1, 11, 434); \
    prod = prod + (YN(2) * (YO(25) * RCT(0, 0))); \
    loss = loss + RCT(0, 1); \
    prod = prod + (YN(13) * (YN(10) * RCS(75))); \
    loss = loss + (YN(2) * RCS(74)); \
    prod = prod + (YN(0) * (YO(25) * RCS(77))); \
    loss = loss + (YN(2) * RCS(76)); \
    prod = prod + (YN(11) * (YN(10) * RCS(79))); \
    loss = loss + (YN(3) * RCS(78)); \
    prod = prod + (YN(5) * (YO(25) * RCS(81))); \
    loss = loss + (YN(4) * RCS(80)); \
    prod = prod + (YN(11) * ((YN(8) * YN(4)) * RCS(83))); \
    loss = loss + (YN(1) * RCS(82)); \
    prod = prod + (YN(18) * ((YN(8) * YN(2)) * RCS(85))); \
    loss = loss + (YN(13) * RCS(84)); \
    prod = prod + (YN(11) * ((YN(10) * YN(4)) * RCS(87))); \
    loss = loss + (YN(6) * RCS(86)); \
    prod = prod + (YN(1) * (YO(31) * RCS(89))); \
    loss = loss + (YN(6) * RCS(88)); \
    prod = prod + (YN(13) * (YN(8) * RCT(0, 2))); \
    loss = loss + RCT(0, 3); \
    prod = prod + (YN(4) * (YO(31) * RCS(92))); \
    loss = loss + (YN(5) * RCS(93)); \
    prod = prod + (YN(3) * (YO(31) * RCS(96))); \
    loss = loss + (YN(4) * RCS(97)); \
    prod = prod + (YN(2) * (YO(31) * RCS(100))); \
    loss = loss + (YN(0) * RCS(101)); \
    prod = prod + (YN(13) * (YO(31) * RCS(104))); \
    loss = loss + (YN(12) * RCS(105)); \
    prod = prod + (YN(6) * (YO(31) * RCS(108))); \
    loss = loss + (YN(7) * RCS(109)); \
    rhs1 = rho * Y0S(1) + dt * WM(23) * (prod + extra); \
    rhs2 = -(dt * WM(23) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(23) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(23) - fnew); \
    UC_UPDATE_TAIL(23); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 25); \
    prod = (YN(16) * (YN(6) * RCT(0, 4))); \
    extra = 0.0; \
    loss = (YN(4) * RCT(0, 5)); \
    prod = prod + (YN(13) * ((YN(8) * YN(7)) * RCS(9))); \
    loss = loss + (YN(6) * RCS(8)); \
    rhs1 = rho * Y0S(0) + dt * WM(24) * (prod + extra); \
    rhs2 = -(dt * WM(24) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(24) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(24) - fnew); \
    UC_UPDATE_TAIL(24); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 26); \
    prod = (YN(21) * (YN(4) * RCS(18))); \
    extra = 0.0; \
    loss = (YN(2) * RCS(19)); \
    prod = prod + (YN(13) * (YN(8) * RCS(23))); \
    loss = loss + (YN(2) * RCS(22)); \
    prod = prod + (YN(14) * (YN(9) * RCS(25))); \
    loss = loss + (YN(3) * RCS(24)); \
    prod = prod + (YN(4) * (YO(26) * RCS(27))); \
    loss = loss + (YN(3) * RCS(26)); \
    prod = prod + (YN(18) * (YN(8) * RCS(29))); \
    loss = loss + (YN(13) * RCS(28)); \
    prod = prod + (YN(8) * (YO(28) * RCS(59))); \
    loss = loss + (YN(4) * RCS(58)); \
    prod = prod + (YN(23) * RCT(0, 1)); \
    loss = loss + (YN(2) * RCT(0, 0)); \
    prod = prod + (YN(23) * (YN(2) * RCS(76))); \
    loss = loss + (YN(0) * RCS(77)); \
    prod = prod + (YN(23) * (YN(4) * RCS(80))); \
    loss = loss + (YN(5) * RCS(81)); \
    prod = prod + (YN(1) * (YO(37) * RCS(176))); \
    loss = loss + (YN(10) * RCS(177)); \
    prod = prod + (YN(3) * (YO(39) * RCS(196))); \
    loss = loss + ((YN(13) * YN(2)) * RCS(197)); \
    rhs1 = rho * Y0S(1) + dt * WM(25) * (prod + extra); \
    rhs2 = -(dt * WM(25) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(25) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(25) - fnew); \
    UC_UPDATE_TAIL(25); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 27); \
    prod = (YN(21) * (YN(3) * RCS(12))); \
    extra = 0.0; \
    loss = (YN(2) * RCS(13)); \
    prod = prod + (YN(25) * (YN(3) * RCS(26))); \
    loss = loss + (YN(4) * RCS(27)); \
    prod = prod + (YN(15) * (YN(8) * RCS(31))); \
    loss = loss + (YN(2) * RCS(30)); \
    prod = prod + (YN(10) * ((YN(8) * YN(2)) * RCS(33))); \
    loss = loss + (YN(4) * RCS(32)); \
    prod = prod + (YN(8) * ((YOS(6) * YN(2)) * RCS(35))); \
    loss = loss + (YN(3) * RCS(34)); \
    prod = prod + (YN(8) * ((YOS(6) * YN(4)) * RCS(37))); \
    loss = loss + (YN(1) * RCS(36)); \
    prod = prod + (YN(9) * ((YN(8) * YN(2)) * RCS(39))); \
    loss = loss + (YN(1) * RCS(38)); \
    prod = prod + (YN(4) * (YO(27) * RCS(40))); \
    loss = loss + (YN(2) * RCS(41)); \
    prod = prod + (YN(1) * (YO(27) * RCS(44))); \
    loss = loss + (YN(3) * RCS(45)); \
    prod = prod + (YN(3) * (YO(36) * RCS(170))); \
    loss = loss + (YN(13) * RCS(171)); \
    rhs1 = rho * Y0S(0) + dt * WM(26) * (prod + extra); \
    rhs2 = -(dt * WM(26) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(26) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(26) - fnew); \
    UC_UPDATE_TAIL(26); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 28); \
    prod = (YN(21) * (YN(4) * RCS(20))); \
    extra = 0.0; \
    loss = (YN(5) * RCS(21)); \
    prod = prod + (YN(26) * (YN(2) * RCS(41))); \
    loss = loss + (YN(4) * RCS(40)); \
    prod = prod + (YN(20) * (YN(8) * RCS(43))); \
    loss = loss + (YN(3) * RCS(42)); \
    prod = prod + (YN(26) * (YN(3) * RCS(45))); \
    loss = loss + (YN(1) * RCS(44)); \
    prod = prod + (YN(20) * (YN(9) * RCS(47))); \
    loss = loss + (YN(1) * RCS(46)); \
    prod = prod + (YN(10) * (YN(8) * RCS(49))); \
    loss = loss + (YN(1) * RCS(48)); \
    rhs1 = rho * Y0S(1) + dt * WM(27) * (prod + extra); \
    rhs2 = -(dt * WM(27) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(27) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(27) - fnew); \
    UC_UPDATE_TAIL(27); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 29); \
    prod = (YN(11) * (YN(0) * RCS(51))); \
    extra = 0.0; \
    loss = (YN(2) * RCS(50)); \
    prod = prod + (YN(13) * (YN(4) * RCS(53))); \
    loss = loss + (YN(2) * RCS(52)); \
    prod = prod + (YN(11) * (YN(5) * RCS(55))); \
    loss = loss + (YN(4) * RCS(54)); \
    prod = prod + (YN(11) * (YN(6) * RCS(57))); \
    loss = loss + (YN(1) * RCS(56)); \
    prod = prod + (YN(11) * (YN(2) * RCT(0, 6))); \
    loss = loss + RCT(0, 7); \
    prod = prod + (YN(17) * RCT(0, 8)); \
    loss = loss + RCT(0, 9); \
    prod = prod + (YN(25) * (YN(4) * RCS(58))); \
    loss = loss + (YN(8) * RCS(59)); \
    prod = prod + (YN(4) * (YO(29) * RCS(60))); \
    loss = loss + (YN(5) * RCS(61)); \
    prod = prod + (YN(2) * (YO(29) * RCS(64))); \
    loss = loss + (YN(0) * RCS(65)); \
    prod = prod + (YN(3) * (YO(29) * RCS(68))); \
    loss = loss + (YN(4) * RCS(69)); \
    prod = prod + (YN(6) * (YO(29) * RCS(70))); \
    loss = loss + (YN(7) * RCS(71)); \
    prod = prod + (YN(1) * (YO(29) * RCS(72))); \
    loss = loss + (YN(6) * RCS(73)); \
    prod = prod + (YO(30) * RCT(0, 10)); \
    loss = loss + (YN(13) * RCT(0, 11)); \
    prod = prod + (YN(2) * (YO(35) * RCS(148))); \
    loss = loss + (YN(13) * RCS(149)); \
    prod = prod + (YN(2) * (YO(32) * RCS(160))); \
    loss = loss + (YN(13) * RCS(161)); \
    rhs1 = rho * Y0S(0) + dt * WM(28) * (prod + extra); \
    rhs2 = -(dt * WM(28) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(28) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(28) - fnew); \
    UC_UPDATE_TAIL(28); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 30); \
    prod = (YN(28) * (YN(5) * RCS(61))); \
    extra = 0.0; \
    loss = (YN(4) * RCS(60)); \
    prod = prod + (YN(17) * (YN(5) * RCS(63))); \
    loss = loss + (YN(4) * RCS(62)); \
    prod = prod + (YN(28) * (YN(0) * RCS(65))); \
    loss = loss + (YN(2) * RCS(64)); \
    prod = prod + (YN(17) * (YN(0) * RCS(67))); \
    loss = loss + (YN(2) * RCS(66)); \
    prod = prod + (YN(28) * (YN(4) * RCS(69))); \
    loss = loss + (YN(3) * RCS(68)); \
    prod = prod + (YN(28) * (YN(7) * RCS(71))); \
    loss = loss + (YN(6) * RCS(70)); \
    prod = prod + (YN(28) * (YN(6) * RCS(73))); \
    loss = loss + (YN(1) * RCS(72)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 420); \
    TM_LD(0, 1, 422); \
    TM_LD(0, 2, 410); \
    TM_LD(0, 3, 408); \
    TM_LD(0, 4, 426); \
    TM_LD(0, 5, 424); \
    TM_LD(0, 6, 430); \
    TM_LD(0, 7, 428); \
    TM_LD(0, 8, 436); \
    TM_LD(0, 9, 438); \
    TM_LD(0, 10, 442); \
    TM_LD(0, 11, 440); \
    prod = prod + (YN(13) * (YN(4) * RCT(1, 0))); \
    loss = loss + RCT(1, 1); \
    rhs1 = rho * Y0S(1) + dt * WM(29) * (prod + extra); \
    rhs2 = -(dt * WM(29) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(29) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(29) - fnew); \
    UC_UPDATE_TAIL(29); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 31); \
    prod = (YN(28) * (YN(13) * RCT(1, 2))); \
    extra = 0.0; \
    loss = RCT(1, 3); \
    prod = prod + (YN(16) * (YN(5) * RCT(1, 4))); \
    loss = loss + RCT(1, 5); \
    prod = prod + (YN(5) * (YO(33) * RCS(113))); \
    loss = loss + (YN(4) * RCS(112)); \
    prod = prod + (YN(5) * (YO(32) * RCS(115))); \
    loss = loss + (YN(4) * RCS(114)); \
    prod = prod + (YN(5) * (YO(35) * RCS(117))); \
    loss = loss + (YN(4) * RCS(116)); \
    prod = prod + (YN(0) * (YO(33) * RCS(119))); \
    loss = loss + (YN(2) * RCS(118)); \
    prod = prod + (YN(0) * (YO(32) * RCS(121))); \
    loss = loss + (YN(2) * RCS(120)); \
    prod = prod + (YN(0) * (YO(35) * RCS(123))); \
    loss = loss + (YN(2) * RCS(122)); \
    prod = prod + (YN(4) * (YO(33) * RCS(125))); \
    loss = loss + (YN(3) * RCS(124)); \
    prod = prod + (YN(4) * (YO(32) * RCS(127))); \
    loss = loss + (YN(3) * RCS(126)); \
    prod = prod + (YN(4) * (YO(35) * RCS(129))); \
    loss = loss + (YN(3) * RCS(128)); \
    prod = prod + (YN(12) * (YO(33) * RCS(131))); \
    loss = loss + (YN(13) * RCS(130)); \
    prod = prod + (YN(12) * (YO(32) * RCS(133))); \
    loss = loss + (YN(13) * RCS(132)); \
    prod = prod + (YN(12) * (YO(35) * RCS(135))); \
    loss = loss + (YN(13) * RCS(134)); \
    prod = prod + (YN(7) * (YO(32) * RCS(137))); \
    loss = loss + (YN(6) * RCS(136)); \
    prod = prod + (YN(7) * (YO(33) * RCS(139))); \
    loss = loss + (YN(6) * RCS(138)); \
    prod = prod + (YN(7) * (YO(35) * RCS(141))); \
    loss = loss + (YN(6) * RCS(140)); \
    rhs1 = rho * Y0S(0) + dt * WM(30) * (prod + extra); \
    rhs2 = -(dt * WM(30) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(30) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(30) - fnew); \
    UC_UPDATE_TAIL(30); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 32); \
    prod = (YN(23) * (YN(6) * RCS(88))); \
    extra = 0.0; \
    loss = (YN(1) * RCS(89)); \
    prod = prod + (YN(13) * (YN(10) * RCT(1, 6))); \
    loss = loss + RCT(1, 7); \
    prod = prod + (YN(5) * (YO(34) * RCS(91))); \
    loss = loss + (YN(4) * RCS(90)); \
    prod = prod + (YN(23) * (YN(5) * RCS(93))); \
    loss = loss + (YN(4) * RCS(92)); \
    prod = prod + (YN(4) * (YO(34) * RCS(95))); \
    loss = loss + (YN(3) * RCS(94)); \
    prod = prod + (YN(23) * (YN(4) * RCS(97))); \
    loss = loss + (YN(3) * RCS(96)); \
    prod = prod + (YN(0) * (YO(34) * RCS(99))); \
    loss = loss + (YN(2) * RCS(98)); \
    prod = prod + (YN(23) * (YN(0) * RCS(101))); \
    loss = loss + (YN(2) * RCS(100)); \
    prod = prod + (YN(12) * (YO(34) * RCS(103))); \
    loss = loss + (YN(13) * RCS(102)); \
    prod = prod + (YN(23) * (YN(12) * RCS(105))); \
    loss = loss + (YN(13) * RCS(104)); \
    prod = prod + (YN(7) * (YO(34) * RCS(107))); \
    loss = loss + (YN(6) * RCS(106)); \
    prod = prod + (YN(23) * (YN(7) * RCS(109))); \
    loss = loss + (YN(6) * RCS(108)); \
    prod = prod + (YN(6) * (YO(34) * RCS(111))); \
    loss = loss + (YN(1) * RCS(110)); \
    prod = prod + (YO(35) * RCT(1, 8)); \
    loss = loss + (YN(2) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(35) * RCS(144))); \
    loss = loss + (YN(6) * RCS(145)); \
    prod = prod + (YN(4) * (YO(35) * RCS(152))); \
    loss = loss + (YN(5) * RCS(153)); \
    prod = prod + (YN(1) * (YO(32) * RCS(154))); \
    loss = loss + (YN(6) * RCS(155)); \
    prod = prod + (YN(3) * (YO(32) * RCS(156))); \
    loss = loss + (YN(4) * RCS(157)); \
    prod = prod + (YN(6) * (YO(32) * RCS(162))); \
    loss = loss + ((YN(4) * YN(4)) * RCS(163)); \
    prod = prod + (YN(4) * (YO(32) * RCS(164))); \
    loss = loss + (YN(5) * RCS(165)); \
    prod = prod + (YO(32) * RCT(1, 10)); \
    loss = loss + (YN(2) * RCT(1, 11)); \
    rhs1 = rho * Y0S(1) + dt * WM(31) * (prod + extra); \
    rhs2 = -(dt * WM(31) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(31) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(31) - fnew); \
    UC_UPDATE_TAIL(31); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 33); \
    prod = (YN(30) * (YN(4) * RCS(114))); \
    extra = 0.0; \
    loss = (YN(5) * RCS(115)); \
    prod = prod + (YN(30) * (YN(2) * RCS(120))); \
    loss = loss + (YN(0) * RCS(121)); \
    prod = prod + (YN(30) * (YN(3) * RCS(126))); \
    loss = loss + (YN(4) * RCS(127)); \
    prod = prod + (YN(30) * (YN(13) * RCS(132))); \
    loss = loss + (YN(12) * RCS(133)); \
    prod = prod + (YN(30) * (YN(6) * RCS(136))); \
    loss = loss + (YN(7) * RCS(137)); \
    prod = prod + (YN(31) * (YN(6) * RCS(155))); \
    loss = loss + (YN(1) * RCS(154)); \
    prod = prod + (YN(31) * (YN(4) * RCS(157))); \
    loss = loss + (YN(3) * RCS(156)); \
    prod = prod + (YN(16) * (YN(5) * RCS(159))); \
    loss = loss + (YN(2) * RCS(158)); \
    prod = prod + (YN(28) * (YN(13) * RCS(161))); \
    loss = loss + (YN(2) * RCS(160)); \
    prod = prod + (YN(31) * ((YN(4) * YN(4)) * RCS(163))); \
    loss = loss + (YN(6) * RCS(162)); \
    prod = prod + (YN(31) * (YN(5) * RCS(165))); \
    loss = loss + (YN(4) * RCS(164)); \
    prod = prod + (YN(31) * (YN(2) * RCT(1, 11))); \
    loss = loss + RCT(1, 10); \
    rhs1 = rho * Y0S(0) + dt * WM(32) * (prod + extra); \
    rhs2 = -(dt * WM(32) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(32) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(32) - fnew); \
    UC_UPDATE_TAIL(32); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 34); \
    prod = (YN(30) * (YN(4) * RCS(112))); \
    extra = 0.0; \
    loss = (YN(5) * RCS(113)); \
    prod = prod + (YN(30) * (YN(2) * RCS(118))); \
    loss = loss + (YN(0) * RCS(119)); \
    prod = prod + (YN(30) * (YN(3) * RCS(124))); \
    loss = loss + (YN(4) * RCS(125)); \
    prod = prod + (YN(30) * (YN(13) * RCS(130))); \
    loss = loss + (YN(12) * RCS(131)); \
    prod = prod + (YN(30) * (YN(6) * RCS(138))); \
    loss = loss + (YN(7) * RCS(139)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 492); \
    TM_LD(1, 1, 494); \
    TM_LD(1, 2, 438); \
    TM_LD(1, 3, 436); \
    TM_LD(1, 4, 486); \
    TM_LD(1, 5, 484); \
    TM_LD(1, 6, 440); \
    TM_LD(1, 7, 442); \
    TM_LD(1, 8, 444); \
    TM_LD(1, 9, 446); \
    TM_LD(1, 10, 450); \
    TM_LD(1, 11, 448); \
    prod = prod + (YN(16) * (YN(4) * RCT(0, 0))); \
    loss = loss + RCT(0, 1); \
    rhs1 = rho * Y0S(1) + dt * WM(33) * (prod + extra); \
    rhs2 = -(dt * WM(33) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(33) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(33) - fnew); \
    UC_UPDATE_TAIL(33); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 35); \
    prod = (YN(13) * (YN(8) * RCT(0, 2))); \
    extra = 0.0; \
    loss = RCT(0, 3); \
    prod = prod + (YN(31) * (YN(4) * RCS(90))); \
    loss = loss + (YN(5) * RCS(91)); \
    prod = prod + (YN(31) * (YN(3) * RCS(94))); \
    loss = loss + (YN(4) * RCS(95)); \
    prod = prod + (YN(31) * (YN(2) * RCS(98))); \
    loss = loss + (YN(0) * RCS(99)); \
    prod = prod + (YN(31) * (YN(13) * RCS(102))); \
    loss = loss + (YN(12) * RCS(103)); \
    prod = prod + (YN(31) * (YN(6) * RCS(106))); \
    loss = loss + (YN(7) * RCS(107)); \
    prod = prod + (YN(31) * (YN(1) * RCS(110))); \
    loss = loss + (YN(6) * RCS(111)); \
    rhs1 = rho * Y0S(0) + dt * WM(34) * (prod + extra); \
    rhs2 = -(dt * WM(34) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(34) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(34) - fnew); \
    UC_UPDATE_TAIL(34); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 36); \
    prod = (YN(30) * (YN(4) * RCS(116))); \
    extra = 0.0; \
    loss = (YN(5) * RCS(117)); \
    prod = prod + (YN(30) * (YN(2) * RCS(122))); \
    loss = loss + (YN(0) * RCS(123)); \
    prod = prod + (YN(30) * (YN(3) * RCS(128))); \
    loss = loss + (YN(4) * RCS(129)); \
    prod = prod + (YN(30) * (YN(13) * RCS(134))); \
    loss = loss + (YN(12) * RCS(135)); \
    prod = prod + (YN(30) * (YN(6) * RCS(140))); \
    loss = loss + (YN(7) * RCS(141)); \
    prod = prod + (YN(18) * (YN(6) * RCS(142))); \
    loss = loss + (YN(4) * RCS(143)); \
    prod = prod + (YN(31) * (YN(2) * RCT(0, 4))); \
    loss = loss + RCT(0, 5); \
    prod = prod + (YN(13) * (YN(11) * RCT(0, 6))); \
    loss = loss + RCT(0, 7); \
    prod = prod + (YN(31) * (YN(6) * RCS(145))); \
    loss = loss + (YN(1) * RCS(144)); \
    prod = prod + (YN(18) * (YN(9) * RCS(147))); \
    loss = loss + (YN(8) * RCS(146)); \
    prod = prod + (YN(28) * (YN(13) * RCS(149))); \
    loss = loss + (YN(2) * RCS(148)); \
    prod = prod + (YN(16) * (YN(5) * RCS(151))); \
    loss = loss + (YN(2) * RCS(150)); \
    prod = prod + (YN(31) * (YN(5) * RCS(153))); \
    loss = loss + (YN(4) * RCS(152)); \
    rhs1 = rho * Y0S(1) + dt * WM(35) * (prod + extra); \
    rhs2 = -(dt * WM(35) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(35) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(35) - fnew); \
    UC_UPDATE_TAIL(35); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 37); \
    prod = (YN(16) * (YN(8) * RCS(167))); \
    extra = 0.0; \
    loss = (YN(3) * RCS(166)); \
    prod = prod + (YN(21) * (YN(13) * RCS(168))); \
    loss = loss + (YN(2) * RCS(169)); \
    prod = prod + (YN(26) * (YN(13) * RCS(171))); \
    loss = loss + (YN(3) * RCS(170)); \
    prod = prod + (YN(2) * (YO(37) * RCT(0, 8))); \
    loss = loss + RCT(0, 9); \
    prod = prod + (YN(6) * (YO(37) * RCS(172))); \
    loss = loss + (YN(1) * RCS(173)); \
    prod = prod + (YN(5) * (YO(37) * RCS(175))); \
    loss = loss + (YN(4) * RCS(174)); \
    prod = prod + (YO(38) * RCT(0, 10)); \
    loss = loss + (YN(2) * RCT(0, 11)); \
    prod = prod + (YN(2) * (YO(38) * RCS(178))); \
    loss = loss + (YN(0) * RCS(179)); \
    prod = prod + (YN(1) * (YO(38) * RCS(180))); \
    loss = loss + (YN(6) * RCS(181)); \
    prod = prod + (YN(13) * (YO(38) * RCS(182))); \
    loss = loss + (YN(12) * RCS(183)); \
    prod = prod + (YN(4) * (YO(38) * RCS(184))); \
    loss = loss + (YN(5) * RCS(185)); \
    prod = prod + (YN(10) * (YO(37) * RCS(186))); \
    loss = loss + (YN(8) * RCS(187)); \
    prod = prod + (YN(13) * ((YN(10) * YN(8)) * RCS(191))); \
    loss = loss + (YN(1) * RCS(190)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 496); \
    TM_LD(0, 1, 498); \
    TM_LD(0, 2, 500); \
    TM_LD(0, 3, 502); \
    TM_LD(0, 4, 508); \
    TM_LD(0, 5, 510); \
    TM_LD(0, 6, 448); \
    TM_LD(0, 7, 450); \
    TM_LD(0, 8, 452); \
    TM_LD(0, 9, 454); \
    TM_LD(0, 10, 466); \
    TM_LD(0, 11, 464); \
    prod = prod + (YO(45) * RCT(1, 0)); \
    loss = loss + (YN(16) * RCT(1, 1)); \
    prod = prod + (YN(1) * (YO(45) * RCS(244))); \
    loss = loss + ((YN(22) * YN(6)) * RCS(245)); \
    prod = prod + (YN(6) * (YO(45) * RCS(248))); \
    loss = loss + ((YN(22) * YN(7)) * RCS(249)); \
    rhs1 = rho * Y0S(0) + dt * WM(36) * (prod + extra); \
    rhs2 = -(dt * WM(36) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(36) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(36) - fnew); \
    UC_UPDATE_TAIL(36); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 38); \
    prod = (YN(36) * RCT(1, 2)); \
    extra = 0.0; \
    loss = (YN(2) * RCT(1, 3)); \
    prod = prod + (YN(36) * (YN(1) * RCS(173))); \
    loss = loss + (YN(6) * RCS(172)); \
    prod = prod + (YN(36) * (YN(4) * RCS(174))); \
    loss = loss + (YN(5) * RCS(175)); \
    prod = prod + (YN(25) * (YN(10) * RCS(177))); \
    loss = loss + (YN(1) * RCS(176)); \
    prod = prod + (YN(36) * (YN(8) * RCS(187))); \
    loss = loss + (YN(10) * RCS(186)); \
    prod = prod + (YN(22) * ((YN(4) * YN(8)) * RCS(189))); \
    loss = loss + (YN(6) * RCS(188)); \
    prod = prod + (YO(43) * RCT(1, 4)); \
    loss = loss + (YN(13) * RCT(1, 5)); \
    rhs1 = rho * Y0S(1) + dt * WM(37) * (prod + extra); \
    rhs2 = -(dt * WM(37) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(37) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(37) - fnew); \
    UC_UPDATE_TAIL(37); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 39); \
    prod = (YN(36) * (YN(2) * RCT(1, 6))); \
    extra = 0.0; \
    loss = RCT(1, 7); \
    prod = prod + (YN(36) * (YN(0) * RCS(179))); \
    loss = loss + (YN(2) * RCS(178)); \
    prod = prod + (YN(36) * (YN(6) * RCS(181))); \
    loss = loss + (YN(1) * RCS(180)); \
    prod = prod + (YN(36) * (YN(12) * RCS(183))); \
    loss = loss + (YN(13) * RCS(182)); \
    prod = prod + (YN(21) * (YN(13) * RCT(1, 8))); \
    loss = loss + RCT(1, 9); \
    prod = prod + (YN(36) * (YN(5) * RCS(185))); \
    loss = loss + (YN(4) * RCS(184)); \
    prod = prod + (YN(4) * (YO(39) * RCS(194))); \
    loss = loss + (YN(5) * RCS(195)); \
    prod = prod + (YN(2) * (YO(39) * RCS(198))); \
    loss = loss + (YN(0) * RCS(199)); \
    prod = prod + (YO(39) * RCT(1, 10)); \
    loss = loss + (YN(2) * RCT(1, 11)); \
    prod = prod + (YN(1) * (YO(39) * RCS(201))); \
    loss = loss + (YN(6) * RCS(200)); \
    prod = prod + (YN(22) * ((YN(4) * YN(11)) * RCS(203))); \
    loss = loss + (YN(6) * RCS(202)); \
    prod = prod + (YN(22) * (YN(13) * RCS(206))); \
    loss = loss + (YN(2) * RCS(207)); \
    prod = prod + (YN(4) * (YO(43) * RCS(238))); \
    loss = loss + ((YO(44) * YN(2)) * RCS(239)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 474); \
    TM_LD(1, 1, 472); \
    TM_LD(1, 2, 488); \
    TM_LD(1, 3, 490); \
    TM_LD(1, 4, 504); \
    TM_LD(1, 5, 506); \
    TM_LD(1, 6, 458); \
    TM_LD(1, 7, 456); \
    TM_LD(1, 8, 462); \
    TM_LD(1, 9, 460); \
    TM_LD(1, 10, 464); \
    TM_LD(1, 11, 466); \
    prod = prod + (YO(45) * RCT(0, 0)); \
    loss = loss + (YN(22) * RCT(0, 1)); \
    prod = prod + (YN(1) * (YO(45) * RCS(242))); \
    loss = loss + ((YN(21) * YN(6)) * RCS(243)); \
    prod = prod + (YN(6) * (YO(45) * RCS(246))); \
    loss = loss + ((YN(21) * YN(7)) * RCS(247)); \
    prod = prod + (YO(48) * RCT(0, 2)); \
    loss = loss + (YN(18) * RCT(0, 3)); \
    prod = prod + (YN(2) * (YO(48) * RCS(269))); \
    loss = loss + ((YN(0) * YN(16)) * RCS(270)); \
    prod = prod + (YO(47) * RCT(0, 4)); \
    loss = loss + (YN(13) * RCT(0, 5)); \
    rhs1 = rho * Y0S(0) + dt * WM(38) * (prod + extra); \
    rhs2 = -(dt * WM(38) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(38) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(38) - fnew); \
    UC_UPDATE_TAIL(38); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 40); \
    prod = (YN(18) * (YN(10) * RCS(193))); \
    extra = (1.0 * (YN(2) * (YO(46) * RCS(251)))); \
    loss = (YN(3) * RCS(192)); \
    prod = prod + (YN(38) * (YN(5) * RCS(195))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(259)))); \
    loss = loss + (YN(4) * RCS(194)); \
    prod = prod + (YN(25) * ((YN(13) * YN(2)) * RCS(197))); \
    loss = loss + (YN(3) * RCS(196)); \
    prod = prod + (YN(38) * (YN(0) * RCS(199))); \
    loss = loss + (YN(2) * RCS(198)); \
    prod = prod + (YN(38) * (YN(2) * RCT(0, 6))); \
    loss = loss + RCT(0, 7); \
    prod = prod + (YN(38) * (YN(6) * RCS(200))); \
    loss = loss + (YN(1) * RCS(201)); \
    prod = prod + (YN(22) * (YN(13) * RCT(0, 8))); \
    loss = loss + RCT(0, 9); \
    prod = prod + (YN(16) * (YN(13) * RCS(205))); \
    loss = loss + (YN(2) * RCS(204)); \
    prod = prod + (YO(41) * RCT(0, 10)); \
    loss = loss + (YN(2) * RCT(0, 11)); \
    prod = prod + (YN(1) * (YO(41) * RCS(228))); \
    loss = loss + (YN(6) * RCS(229)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 470); \
    TM_LD(0, 1, 468); \
    TM_LD(0, 2, 472); \
    TM_LD(0, 3, 474); \
    TM_LD(0, 4, 478); \
    TM_LD(0, 5, 476); \
    TM_LD(0, 6, 480); \
    TM_LD(0, 7, 482); \
    TM_LD(0, 8, 484); \
    TM_LD(0, 9, 486); \
    TM_LD(0, 10, 490); \
    TM_LD(0, 11, 488); \
    prod = prod + (YO(42) * RCT(1, 0)); \
    loss = loss + (YN(2) * RCT(1, 1)); \
    prod = prod + (YN(1) * (YO(42) * RCS(230))); \
    loss = loss + (YN(6) * RCS(231)); \
    prod = prod + (YO(45) * RCT(1, 2)); \
    loss = loss + (YN(21) * RCT(1, 3)); \
    prod = prod + (YO(48) * RCT(1, 4)); \
    loss = loss + (YN(16) * RCT(1, 5)); \
    prod = prod + (YN(4) * (YO(48) * RCS(261))); \
    loss = loss + ((YN(5) * YN(22)) * RCS(262)); \
    prod = prod + (YN(2) * (YO(48) * RCS(263))); \
    loss = loss + ((YN(0) * YN(22)) * RCS(264)); \
    prod = prod + (YN(2) * (YO(48) * RCS(267))); \
    loss = loss + (YN(18) * RCS(268)); \
    prod = prod + (YN(2) * (YO(47) * RCS(275))); \
    loss = loss + (YN(13) * RCS(276)); \
    rhs1 = rho * Y0S(1) + dt * WM(39) * (prod + extra); \
    rhs2 = -(dt * WM(39) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(39) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(39) - fnew); \
    UC_UPDATE_TAIL(39); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 41); \
    prod = (YN(18) * (YN(13) * RCT(1, 6))); \
    extra = 0.0; \
    loss = RCT(1, 7); \
    prod = prod + (YN(6) * (YO(41) * RCS(209))); \
    loss = loss + (YN(1) * RCS(208)); \
    prod = prod + (YN(6) * (YO(42) * RCS(211))); \
    loss = loss + (YN(1) * RCS(210)); \
    prod = prod + (YN(0) * (YO(41) * RCS(213))); \
    loss = loss + (YN(2) * RCS(212)); \
    prod = prod + (YN(0) * (YO(42) * RCS(215))); \
    loss = loss + (YN(2) * RCS(214)); \
    prod = prod + (YN(4) * (YO(41) * RCS(217))); \
    loss = loss + (YN(3) * RCS(216)); \
    prod = prod + (YN(4) * (YO(42) * RCS(219))); \
    loss = loss + (YN(3) * RCS(218)); \
    prod = prod + (YN(5) * (YO(42) * RCS(221))); \
    loss = loss + (YN(4) * RCS(220)); \
    prod = prod + (YN(5) * (YO(41) * RCS(223))); \
    loss = loss + (YN(4) * RCS(222)); \
    prod = prod + (YN(7) * (YO(41) * RCS(225))); \
    loss = loss + (YN(6) * RCS(224)); \
    prod = prod + (YN(7) * (YO(42) * RCS(227))); \
    loss = loss + (YN(6) * RCS(226)); \
    rhs1 = rho * Y0S(0) + dt * WM(40) * (prod + extra); \
    rhs2 = -(dt * WM(40) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(40) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(40) - fnew); \
    UC_UPDATE_TAIL(40); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 42); \
    prod = (YN(40) * (YN(1) * RCS(208))); \
    extra = 0.0; \
    loss = (YN(6) * RCS(209)); \
    prod = prod + (YN(40) * (YN(2) * RCS(212))); \
    loss = loss + (YN(0) * RCS(213)); \
    prod = prod + (YN(40) * (YN(3) * RCS(216))); \
    loss = loss + (YN(4) * RCS(217)); \
    prod = prod + (YN(40) * (YN(4) * RCS(222))); \
    loss = loss + (YN(5) * RCS(223)); \
    prod = prod + (YN(40) * (YN(6) * RCS(224))); \
    loss = loss + (YN(7) * RCS(225)); \
    prod = prod + (YO(42) * RCT(1, 8)); \
    loss = loss + RCT(1, 9); \
    prod = prod + (YN(39) * (YN(2) * RCT(1, 10))); \
    loss = loss + RCT(1, 11); \
    prod = prod + (YN(39) * (YN(6) * RCS(229))); \
    loss = loss + (YN(1) * RCS(228)); \
    rhs1 = rho * Y0S(1) + dt * WM(41) * (prod + extra); \
    rhs2 = -(dt * WM(41) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(41) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(41) - fnew); \
    UC_UPDATE_TAIL(41); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 43); \
    prod = (YN(40) * (YN(1) * RCS(210))); \
    extra = 0.0; \
    loss = (YN(6) * RCS(211)); \
    prod = prod + (YN(40) * (YN(2) * RCS(214))); \
    loss = loss + (YN(0) * RCS(215)); \
    prod = prod + (YN(40) * (YN(3) * RCS(218))); \
    loss = loss + (YN(4) * RCS(219)); \
    prod = prod + (YN(40) * (YN(4) * RCS(220))); \
    loss = loss + (YN(5) * RCS(221)); \
    prod = prod + (YN(40) * (YN(6) * RCS(226))); \
    loss = loss + (YN(7) * RCS(227)); \
    prod = prod + (YN(41) * RCT(1, 9)); \
    loss = loss + RCT(1, 8); \
    TM_WAIT(0); \
    TM_LD(1, 0, 494); \
    TM_LD(1, 1, 492); \
    TM_LD(1, 2, 498); \
    TM_LD(1, 3, 496); \
    TM_LD(1, 4, 510); \
    TM_LD(1, 5, 508); \
    TM_LD(1, 6, 502); \
    TM_LD(1, 7, 500); \
    TM_LD(1, 8, 506); \
    TM_LD(1, 9, 504); \
    prod = prod + (YN(16) * (YN(13) * RCT(0, 0))); \
    loss = loss + RCT(0, 1); \
    prod = prod + (YN(39) * (YN(2) * RCT(0, 2))); \
    loss = loss + RCT(0, 3); \
    prod = prod + (YN(39) * (YN(6) * RCS(231))); \
    loss = loss + (YN(1) * RCS(230)); \
    rhs1 = rho * Y0S(0) + dt * WM(42) * (prod + extra); \
    rhs2 = -(dt * WM(42) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(42) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(42) - fnew); \
    UC_UPDATE_TAIL(42); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 44); \
    prod = (YN(22) * ((YN(21) * YN(2)) * RCS(233))); \
    extra = 0.0; \
    loss = RCS(232); \
    prod = prod + (YN(22) * (YOS(7) * RCT(0, 4))); \
    loss = loss + RCT(0, 5); \
    prod = prod + (YN(22) * (YOS(7) * RCT(0, 6))); \
    loss = loss + RCT(0, 7); \
    prod = prod + (YN(22) * (YN(16) * RCS(235))); \
    loss = loss + (YN(2) * RCS(234)); \
    prod = prod + (YN(22) * ((YN(0) * YN(21)) * RCS(237))); \
    loss = loss + (YN(2) * RCS(236)); \
    prod = prod + (YN(38) * ((YO(44) * YN(2)) * RCS(239))); \
    loss = loss + (YN(4) * RCS(238)); \
    prod = prod + (YN(22) * ((YN(12) * YN(21)) * RCS(241))); \
    loss = loss + (YN(13) * RCS(240)); \
    prod = prod + (YN(37) * (YN(13) * RCT(0, 8))); \
    loss = loss + RCT(0, 9); \
    prod = prod + (YN(2) * (YO(48) * RCS(271))); \
    loss = loss + ((YN(0) * YN(13)) * RCS(272)); \
    prod = prod + (YN(4) * (YO(47) * RCS(279))); \
    loss = loss + ((YN(5) * YN(2)) * RCS(280)); \
    rhs1 = rho * Y0S(1) + dt * WM(43) * (prod + extra); \
    rhs2 = -(dt * WM(43) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(43) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(43) - fnew); \
    UC_UPDATE_TAIL(43); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 45); \
    prod = (YN(43) * (YN(4) * RCS(238))); \
    extra = 0.0; \
    loss = ((YN(2) * YN(38)) * RCS(239)); \
    rhs1 = rho * Y0S(0) + dt * WM(44) * (prod + extra); \
    rhs2 = -(dt * WM(44) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(44) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(44) - fnew); \
    UC_UPDATE_TAIL(44); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 46); \
    prod = (YN(39) * (YN(21) * RCT(0, 10))); \
    extra = 0.0; \
    loss = RCT(0, 11); \
    TM_WAIT(1); \
    prod = prod + (YN(36) * (YN(16) * RCT(1, 0))); \
    loss = loss + RCT(1, 1); \
    prod = prod + (YN(38) * (YN(22) * RCT(1, 2))); \
    loss = loss + RCT(1, 3); \
    prod = prod + (YN(38) * ((YN(21) * YN(6)) * RCS(243))); \
    loss = loss + (YN(1) * RCS(242)); \
    prod = prod + (YN(36) * ((YN(22) * YN(6)) * RCS(245))); \
    loss = loss + (YN(1) * RCS(244)); \
    prod = prod + (YN(38) * ((YN(21) * YN(7)) * RCS(247))); \
    loss = loss + (YN(6) * RCS(246)); \
    prod = prod + (YN(36) * ((YN(22) * YN(7)) * RCS(249))); \
    loss = loss + (YN(6) * RCS(248)); \
    rhs1 = rho * Y0S(1) + dt * WM(45) * (prod + extra); \
    rhs2 = -(dt * WM(45) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(45) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(45) - fnew); \
    UC_UPDATE_TAIL(45); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 47); \
    prod = 0.0; \
    extra = 0.0; \
    loss = RCS(250); \
    prod = prod + 0.0; \
    loss = loss + (YN(2) * RCS(251)); \
    prod = prod + 0.0; \
    loss = loss + (YN(2) * RCS(252)); \
    prod = prod + 0.0; \
    loss = loss + (YN(2) * RCS(253)); \
    prod = prod + (YN(18) * ((YN(0) * YO(48)) * RCS(255))); \
    loss = loss + (YN(2) * RCS(254)); \
    prod = prod + (YN(18) * ((YN(5) * YO(48)) * RCS(257))); \
    loss = loss + (YN(4) * RCS(256)); \
    prod = prod + 0.0; \
    loss = loss + (YN(4) * RCS(258)); \
    prod = prod + 0.0; \
    loss = loss + (YN(4) * RCS(259)); \
    prod = prod + 0.0; \
    loss = loss + (YN(4) * RCS(260)); \
    rhs1 = rho * Y0S(0) + dt * WM(46) * (prod + extra); \
    rhs2 = -(dt * WM(46) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(46) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(46) - fnew); \
    UC_UPDATE_TAIL(46); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 48); \
    prod = (YN(38) * (YN(13) * RCT(1, 4))); \
    extra = (1.0 * (YN(46) * (YN(2) * RCS(252)))); \
    loss = RCT(1, 5); \
    prod = prod + (YN(18) * (YN(16) * RCS(274))); \
    extra = extra + (1.0 * (YN(46) * (YN(4) * RCS(258)))); \
    loss = loss + (YN(2) * RCS(273)); \
    prod = prod + (YN(39) * (YN(13) * RCS(276))); \
    loss = loss + (YN(2) * RCS(275)); \
    prod = prod + (YN(22) * ((YN(0) * YN(16)) * RCS(278))); \
    loss = loss + (YN(2) * RCS(277)); \
    prod = prod + (YN(43) * ((YN(5) * YN(2)) * RCS(280))); \
    loss = loss + (YN(4) * RCS(279)); \
    rhs1 = rho * Y0S(1) + dt * WM(47) * (prod + extra); \
    rhs2 = -(dt * WM(47) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(47) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(47) - fnew); \
    UC_UPDATE_TAIL(47); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 49); \
    prod = (YN(46) * (YN(2) * RCS(254))); \
    extra = 0.0; \
    loss = ((YN(0) * YN(18)) * RCS(255)); \
    prod = prod + (YN(46) * (YN(4) * RCS(256))); \
    loss = loss + ((YN(5) * YN(18)) * RCS(257)); \
    prod = prod + (YN(38) * (YN(18) * RCT(1, 6))); \
    loss = loss + RCT(1, 7); \
    prod = prod + (YN(39) * (YN(16) * RCT(1, 8))); \
    loss = loss + RCT(1, 9); \
    prod = prod + (YN(39) * ((YN(5) * YN(22)) * RCS(262))); \
    loss = loss + (YN(4) * RCS(261)); \
    prod = prod + (YN(39) * ((YN(0) * YN(22)) * RCS(264))); \
    loss = loss + (YN(2) * RCS(263)); \
    prod = prod + (YN(16) * ((YOS(4) * YN(13)) * RCS(266))); \
    loss = loss + (YN(2) * RCS(265)); \
    prod = prod + (YN(39) * (YN(18) * RCS(268))); \
    loss = loss + (YN(2) * RCS(267)); \
    prod = prod + (YN(38) * ((YN(0) * YN(16)) * RCS(270))); \
    loss = loss + (YN(2) * RCS(269)); \
    prod = prod + (YN(43) * ((YN(0) * YN(13)) * RCS(272))); \
    loss = loss + (YN(2) * RCS(271)); \
    rhs1 = rho * Y0S(0) + dt * WM(48) * (prod + extra); \
    rhs2 = -(dt * WM(48) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(48) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(48) - fnew); \
    UC_UPDATE_TAIL(48); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 50); \
    extra = 0.0; \
    rhs1 = rho * Y0S(1) + dt * WM(49) * (prod + extra); \
    rhs2 = 0.0; \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(49) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(49) - fnew); \
    UC_UPDATE_TAIL(49); \
    UC_TR_SYNC(); \
    extra = 0.0; \
    rhs1 = rho * Y0S(0) + dt * WM(50) * (prod + extra); \
    rhs2 = 0.0; \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(50) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(50) - fnew); \
    UC_UPDATE_TAIL(50); \
    UC_TR_SYNC(); \
} while (0)
#ifdef __CUDACC__
static __constant__ int16_t uc_tr_trow[256] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51, 52, 53, 54, 55, 56, 57, 58, 59, 60, 61, 62, 63, 64, 65, 66, 67, 68, 69, 70, 71, 72, 73, 74, 75, 76, 77, 78, 79, 80, 81, 82, 83, 84, 85, 86, 87, 88, 89, 90, 91, 92, 93, 94, 95, 96, 97, 98, 99, 100, 101, 102, 103, 104, 105, 106, 107, 108, 109, 112, 113, 114, 115, 116, 117, 118, 119, 120, 121, 124, 125, 126, 127, 132, 133, 134, 135, 136, 137, 138, 139, 140, 141, 142, 143, 144, 145, 146, 147, 148, 149, 150, 151, 152, 153, 154, 155, 156, 157, 158, 159, 160, 161, 162, 163, 164, 165, 166, 167, 168, 169, 170, 171, 172, 173, 174, 175, 176, 177, 178, 179, 180, 181, 182, 183, 184, 185, 186, 187, 190, 191, 192, 193, 194, 195, 196, 197, 198, 199, 200, 201, 250, 251, 252, 253, 270, 271, 272, 273, 290, 291, 292, 293, 294, 295, 318, 319, 320, 321, 352, 353, 356, 357, 358, 359, 382, 383, 390, 391, 398, 399, 406, 407, 424, 425, 430, 431, 436, 437, 458, 459, 460, 461, 464, 465, 466, 467, 472, 473, 474, 475, 484, 485, 486, 487, 488, 489, 490, 491, 518, 519, 520, 521, 534, 535};
static __constant__ int16_t uc_tr_srow[281] = {110, 111, 122, 123, 128, 129, 130, 131, 188, 189, 202, 203, 204, 205, 206, 207, 208, 209, 210, 211, 212, 213, 214, 215, 216, 217, 218, 219, 220, 221, 222, 223, 224, 225, 226, 227, 228, 229, 230, 231, 232, 233, 234, 235, 236, 237, 238, 239, 240, 241, 242, 243, 244, 245, 246, 247, 248, 249, 254, 255, 256, 257, 258, 259, 260, 261, 262, 263, 264, 265, 266, 267, 268, 269, 274, 275, 276, 277, 278, 279, 280, 281, 282, 283, 284, 285, 286, 287, 288, 289, 296, 297, 298, 299, 300, 301, 302, 303, 304, 305, 306, 307, 308, 309, 310, 311, 312, 313, 314, 315, 316, 317, 322, 323, 324, 325, 326, 327, 328, 329, 330, 331, 332, 333, 334, 335, 336, 337, 338, 339, 340, 341, 342, 343, 344, 345, 346, 347, 348, 349, 350, 351, 354, 355, 360, 361, 362, 363, 364, 365, 366, 367, 368, 369, 370, 371, 372, 373, 374, 375, 376, 377, 378, 379, 380, 381, 384, 385, 386, 387, 388, 389, 392, 393, 394, 395, 396, 397, 400, 401, 402, 403, 404, 405, 408, 409, 410, 411, 412, 413, 414, 415, 416, 417, 418, 419, 420, 421, 422, 423, 426, 427, 428, 429, 432, 433, 434, 435, 438, 439, 440, 441, 442, 443, 444, 445, 446, 447, 448, 449, 450, 451, 452, 453, 454, 455, 456, 457, 462, 463, 468, 469, 470, 471, 476, 477, 478, 479, 480, 481, 482, 483, 492, 493, 494, 495, 496, 497, 498, 499, 500, 502, 504, 506, 508, 509, 510, 511, 512, 514, 516, 522, 523, 524, 525, 526, 527, 528, 529, 530, 531, 532, 533, 536, 537, 538, 539, 540, 541, 542, 543};
#else
static const short uc_tr_trow[256] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51, 52, 53, 54, 55, 56, 57, 58, 59, 60, 61, 62, 63, 64, 65, 66, 67, 68, 69, 70, 71, 72, 73, 74, 75, 76, 77, 78, 79, 80, 81, 82, 83, 84, 85, 86, 87, 88, 89, 90, 91, 92, 93, 94, 95, 96, 97, 98, 99, 100, 101, 102, 103, 104, 105, 106, 107, 108, 109, 112, 113, 114, 115, 116, 117, 118, 119, 120, 121, 124, 125, 126, 127, 132, 133, 134, 135, 136, 137, 138, 139, 140, 141, 142, 143, 144, 145, 146, 147, 148, 149, 150, 151, 152, 153, 154, 155, 156, 157, 158, 159, 160, 161, 162, 163, 164, 165, 166, 167, 168, 169, 170, 171, 172, 173, 174, 175, 176, 177, 178, 179, 180, 181, 182, 183, 184, 185, 186, 187, 190, 191, 192, 193, 194, 195, 196, 197, 198, 199, 200, 201, 250, 251, 252, 253, 270, 271, 272, 273, 290, 291, 292, 293, 294, 295, 318, 319, 320, 321, 352, 353, 356, 357, 358, 359, 382, 383, 390, 391, 398, 399, 406, 407, 424, 425, 430, 431, 436, 437, 458, 459, 460, 461, 464, 465, 466, 467, 472, 473, 474, 475, 484, 485, 486, 487, 488, 489, 490, 491, 518, 519, 520, 521, 534, 535};
static const short uc_tr_srow[281] = {110, 111, 122, 123, 128, 129, 130, 131, 188, 189, 202, 203, 204, 205, 206, 207, 208, 209, 210, 211, 212, 213, 214, 215, 216, 217, 218, 219, 220, 221, 222, 223, 224, 225, 226, 227, 228, 229, 230, 231, 232, 233, 234, 235, 236, 237, 238, 239, 240, 241, 242, 243, 244, 245, 246, 247, 248, 249, 254, 255, 256, 257, 258, 259, 260, 261, 262, 263, 264, 265, 266, 267, 268, 269, 274, 275, 276, 277, 278, 279, 280, 281, 282, 283, 284, 285, 286, 287, 288, 289, 296, 297, 298, 299, 300, 301, 302, 303, 304, 305, 306, 307, 308, 309, 310, 311, 312, 313, 314, 315, 316, 317, 322, 323, 324, 325, 326, 327, 328, 329, 330, 331, 332, 333, 334, 335, 336, 337, 338, 339, 340, 341, 342, 343, 344, 345, 346, 347, 348, 349, 350, 351, 354, 355, 360, 361, 362, 363, 364, 365, 366, 367, 368, 369, 370, 371, 372, 373, 374, 375, 376, 377, 378, 379, 380, 381, 384, 385, 386, 387, 388, 389, 392, 393, 394, 395, 396, 397, 400, 401, 402, 403, 404, 405, 408, 409, 410, 411, 412, 413, 414, 415, 416, 417, 418, 419, 420, 421, 422, 423, 426, 427, 428, 429, 432, 433, 434, 435, 438, 439, 440, 441, 442, 443, 444, 445, 446, 447, 448, 449, 450, 451, 452, 453, 454, 455, 456, 457, 462, 463, 468, 469, 470, 471, 476, 477, 478, 479, 480, 481, 482, 483, 492, 493, 494, 495, 496, 497, 498, 499, 500, 502, 504, 506, 508, 509, 510, 511, 512, 514, 516, 522, 523, 524, 525, 526, 527, 528, 529, 530, 531, 532, 533, 536, 537, 538, 539, 540, 541, 542, 543};
#endif
