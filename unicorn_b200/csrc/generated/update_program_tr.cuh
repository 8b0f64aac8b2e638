// Generated by unicorn_b200/mech/codegen.py: the in-place species-update program
// (src/lib/solvesp.f:85-2806) for a tile whose RC block is held on chip.
// RC slots 0..255 in tensor memory (slot i in columns 2i, 2i+1: low and high
// word), slots 256..543 in shared memory. Requires RCS(i) (shared-memory row i of the
// cell), TM_LD(bank, q, col) (load the double at column col into slot q of a
// register bank), TM_WAIT(bank) (wait for the loads of that bank), RCT(bank, q),
// UC_TR_PF(slot, k) (fetch Y0, FACE_SUM and FACE_NBR of species k into register slot 0
// or 1; read as Y0S, FSS, FNS), UC_TR_SYNC() (after every species: a barrier or nothing)
// and the accessors of the in-place program (YO, YN, YOS, SOUR, WM, UC_UPDATE_TAIL;
// scalars rho, dt, sor1, sor2, rsd). The production, extra and loss statements of a
// species are interleaved; each sum keeps the reference's order.
// 81 segments and 962 tensor-memory loads per cell and pass.
#pragma once
#define UC_TR_NT 256
#define UC_TR_NS 288
#define UC_TR_SEG 12
#define UC_UPDATE_FLOPS_PER_CELL_PASS 6261
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
    TM_LD(1, 10, 232); \
    TM_LD(1, 11, 234); \
    UC_TR_PF(0, 0); \
    UC_TR_PF(1, 1); \
    prod = ((YO(4) * YO(2)) * RCT(0, 0)); \
    extra = (1.0 * ((YO(46) * YO(2)) * RCS(246))); \
    loss = (YO(3) * RCT(0, 1)); \
    prod = prod + ((YO(5) * YO(2)) * RCT(0, 2)); \
    extra = extra + (1.0 * ((YO(46) * YO(2)) * RCS(248))); \
    loss = loss + (YO(4) * RCT(0, 3)); \
    prod = prod + ((YO(2) * YO(2)) * RCT(0, 4)); \
    extra = extra + (1.0 * ((YO(46) * YO(2)) * RCS(250))); \
    loss = loss + RCT(0, 5); \
    prod = prod + ((YO(6) * YO(2)) * RCT(0, 6)); \
    loss = loss + (YO(1) * RCT(0, 7)); \
    prod = prod + ((YO(7) * YO(2)) * RCT(0, 8)); \
    loss = loss + (YO(6) * RCT(0, 9)); \
    prod = prod + ((YO(10) * YO(2)) * RCT(0, 10)); \
    loss = loss + (YO(8) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 248); \
    TM_LD(0, 1, 250); \
    TM_LD(0, 2, 252); \
    TM_LD(0, 3, 254); \
    TM_LD(0, 4, 280); \
    TM_LD(0, 5, 282); \
    TM_LD(0, 6, 304); \
    TM_LD(0, 7, 306); \
    TM_LD(0, 8, 328); \
    TM_LD(0, 9, 330); \
    TM_LD(0, 10, 348); \
    TM_LD(0, 11, 350); \
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
    TM_LD(1, 0, 384); \
    TM_LD(1, 1, 386); \
    TM_LD(1, 2, 388); \
    TM_LD(1, 3, 390); \
    TM_LD(1, 4, 484); \
    TM_LD(1, 5, 486); \
    TM_LD(1, 6, 2); \
    TM_LD(1, 7, 0); \
    TM_LD(1, 8, 24); \
    TM_LD(1, 9, 26); \
    TM_LD(1, 10, 38); \
    TM_LD(1, 11, 36); \
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
    TM_LD(0, 0, 44); \
    TM_LD(0, 1, 46); \
    TM_LD(0, 2, 52); \
    TM_LD(0, 3, 54); \
    TM_LD(0, 4, 56); \
    TM_LD(0, 5, 58); \
    TM_LD(0, 6, 64); \
    TM_LD(0, 7, 66); \
    TM_LD(0, 8, 94); \
    TM_LD(0, 9, 92); \
    TM_LD(0, 10, 118); \
    TM_LD(0, 11, 116); \
    prod = prod + (YO(16) * RCT(1, 0)); \
    loss = loss + (YO(21) * RCT(1, 1)); \
    prod = prod + ((YO(22) * YO(2)) * RCT(1, 2)); \
    loss = loss + (YO(21) * RCT(1, 3)); \
    prod = prod + ((YO(28) * YO(2)) * RCT(1, 4)); \
    loss = loss + (YO(11) * RCT(1, 5)); \
    prod = prod + ((YO(29) * YO(2)) * RCS(4)); \
    loss = loss + (YO(28) * RCS(5)); \
    prod = prod + ((YO(29) * YO(2)) * RCS(6)); \
    loss = loss + (YO(17) * RCS(7)); \
    prod = prod + ((YO(23) * YO(2)) * RCS(20)); \
    loss = loss + (YO(25) * RCS(21)); \
    prod = prod + ((YO(31) * YO(2)) * RCS(48)); \
    loss = loss + (YO(34) * RCS(49)); \
    prod = prod + ((YO(31) * YO(2)) * RCS(50)); \
    loss = loss + (YO(23) * RCS(51)); \
    prod = prod + ((YO(30) * YO(2)) * RCS(72)); \
    loss = loss + (YO(33) * RCS(73)); \
    prod = prod + ((YO(30) * YO(2)) * RCS(74)); \
    loss = loss + (YO(32) * RCS(75)); \
    prod = prod + ((YO(30) * YO(2)) * RCS(76)); \
    loss = loss + (YO(35) * RCS(77)); \
    prod = prod + ((YO(38) * YO(2)) * RCS(144)); \
    loss = loss + (YO(36) * RCS(145)); \
    prod = prod + ((YO(39) * YO(2)) * RCS(166)); \
    loss = loss + (YO(38) * RCS(167)); \
    prod = prod + ((YO(40) * YO(2)) * RCS(186)); \
    loss = loss + (YO(41) * RCS(187)); \
    prod = prod + ((YO(40) * YO(2)) * RCS(188)); \
    loss = loss + (YO(42) * RCS(189)); \
    prod = prod + ((YO(43) * YO(2)) * RCS(222)); \
    loss = loss + ((YO(21) * YO(22)) * RCS(223)); \
    prod = prod + ((YO(46) * YO(2)) * RCS(252)); \
    loss = loss + ((YO(48) * YO(18)) * RCS(253)); \
    prod = prod + ((YO(48) * YO(2)) * RCS(268)); \
    loss = loss + ((YO(39) * YO(22)) * RCS(269)); \
    prod = prod + ((YO(48) * YO(2)) * RCS(274)); \
    loss = loss + ((YO(16) * YO(38)) * RCS(275)); \
    prod = prod + ((YO(48) * YO(2)) * RCS(276)); \
    loss = loss + ((YO(43) * YO(13)) * RCS(277)); \
    prod = prod + ((YO(47) * YO(2)) * RCS(284)); \
    loss = loss + ((YO(22) * YO(16)) * RCS(285)); \
    prod = prod + (SOUR(0) * YO(21)); \
    rhs1 = rho * Y0S(0) + dt * WM(0) * (prod + extra); \
    rhs2 = -(dt * WM(0) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(0) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(0) - fnew); \
    UC_UPDATE_TAIL(0); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 2); \
    prod = ((YO(4) * YO(3)) * RCT(1, 6)); \
    extra = 0.0; \
    loss = (YO(2) * RCT(1, 7)); \
    prod = prod + ((YO(3) * YO(3)) * RCT(1, 8)); \
    loss = loss + RCT(1, 9); \
    prod = prod + (YO(6) * RCT(1, 10)); \
    loss = loss + (YO(2) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 142); \
    TM_LD(1, 1, 140); \
    TM_LD(1, 2, 162); \
    TM_LD(1, 3, 160); \
    TM_LD(1, 4, 194); \
    TM_LD(1, 5, 192); \
    TM_LD(1, 6, 198); \
    TM_LD(1, 7, 196); \
    TM_LD(1, 8, 222); \
    TM_LD(1, 9, 220); \
    TM_LD(1, 10, 254); \
    TM_LD(1, 11, 252); \
    prod = prod + ((YO(6) * YO(2)) * RCT(0, 0)); \
    loss = loss + (YN(0) * RCT(0, 1)); \
    prod = prod + ((YO(6) * YO(3)) * RCT(0, 2)); \
    loss = loss + (YO(4) * RCT(0, 3)); \
    prod = prod + ((YO(6) * YO(4)) * RCT(0, 4)); \
    loss = loss + (YO(5) * RCT(0, 5)); \
    prod = prod + ((YO(6) * YO(6)) * RCT(0, 6)); \
    loss = loss + (YO(7) * RCT(0, 7)); \
    prod = prod + ((YO(9) * YO(3)) * RCT(0, 8)); \
    loss = loss + (YO(8) * RCT(0, 9)); \
    prod = prod + ((YO(8) * YO(6)) * RCT(0, 10)); \
    loss = loss + (YO(10) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 258); \
    TM_LD(0, 1, 256); \
    TM_LD(0, 2, 270); \
    TM_LD(0, 3, 268); \
    TM_LD(0, 4, 298); \
    TM_LD(0, 5, 296); \
    TM_LD(0, 6, 342); \
    TM_LD(0, 7, 340); \
    TM_LD(0, 8, 370); \
    TM_LD(0, 9, 368); \
    TM_LD(0, 10, 398); \
    TM_LD(0, 11, 396); \
    prod = prod + ((YO(10) * YO(6)) * RCT(1, 0)); \
    loss = loss + (YO(11) * RCT(1, 1)); \
    prod = prod + ((YO(13) * YO(6)) * RCT(1, 2)); \
    loss = loss + (YO(12) * RCT(1, 3)); \
    prod = prod + ((YO(11) * YO(4)) * RCT(1, 4)); \
    loss = loss + (YO(13) * RCT(1, 5)); \
    prod = prod + ((YO(17) * YO(3)) * RCT(1, 6)); \
    loss = loss + (YO(13) * RCT(1, 7)); \
    prod = prod + (((YO(8) * YO(4)) * YO(2)) * RCT(1, 8)); \
    loss = loss + (YO(15) * RCT(1, 9)); \
    prod = prod + (YN(0) * (YO(9) * RCT(1, 10))); \
    loss = loss + (YO(14) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 402); \
    TM_LD(1, 1, 400); \
    TM_LD(1, 2, 406); \
    TM_LD(1, 3, 404); \
    TM_LD(1, 4, 418); \
    TM_LD(1, 5, 416); \
    TM_LD(1, 6, 458); \
    TM_LD(1, 7, 456); \
    TM_LD(1, 8, 462); \
    TM_LD(1, 9, 460); \
    TM_LD(1, 10, 474); \
    TM_LD(1, 11, 472); \
    prod = prod + (((YO(8) * YO(4)) * YO(2)) * RCT(0, 0)); \
    loss = loss + (YO(14) * RCT(0, 1)); \
    prod = prod + ((YO(10) * YO(3)) * RCT(0, 2)); \
    loss = loss + (YO(20) * RCT(0, 3)); \
    prod = prod + ((YO(11) * YO(6)) * RCT(0, 4)); \
    loss = loss + (YO(17) * RCT(0, 5)); \
    prod = prod + ((YO(16) * YO(6)) * RCT(0, 6)); \
    loss = loss + (YO(18) * RCT(0, 7)); \
    prod = prod + ((YO(22) * YO(6)) * RCT(0, 8)); \
    loss = loss + (YO(16) * RCT(0, 9)); \
    prod = prod + ((YO(11) * YO(10)) * RCT(0, 10)); \
    loss = loss + (YO(22) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 478); \
    TM_LD(0, 1, 476); \
    TM_LD(0, 2, 482); \
    TM_LD(0, 3, 480); \
    TM_LD(0, 4, 498); \
    TM_LD(0, 5, 496); \
    TM_LD(0, 6, 2); \
    TM_LD(0, 7, 0); \
    TM_LD(0, 8, 4); \
    TM_LD(0, 9, 6); \
    TM_LD(0, 10, 8); \
    TM_LD(0, 11, 10); \
    prod = prod + ((YO(23) * YO(3)) * RCT(1, 0)); \
    loss = loss + (YO(22) * RCT(1, 1)); \
    prod = prod + ((YO(21) * YO(6)) * RCT(1, 2)); \
    loss = loss + (YO(22) * RCT(1, 3)); \
    prod = prod + ((YO(11) * YO(8)) * RCT(1, 4)); \
    loss = loss + (YO(21) * RCT(1, 5)); \
    prod = prod + (((YO(8) * YO(8)) * YO(4)) * RCT(1, 6)); \
    loss = loss + (YO(26) * RCT(1, 7)); \
    prod = prod + (((YO(9) * YO(8)) * YO(2)) * RCT(1, 8)); \
    loss = loss + (YO(26) * RCT(1, 9)); \
    prod = prod + ((YO(26) * YO(3)) * RCT(1, 10)); \
    loss = loss + (YO(27) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 18); \
    TM_LD(1, 1, 16); \
    TM_LD(1, 2, 22); \
    TM_LD(1, 3, 20); \
    TM_LD(1, 4, 30); \
    TM_LD(1, 5, 28); \
    TM_LD(1, 6, 38); \
    TM_LD(1, 7, 36); \
    TM_LD(1, 8, 42); \
    TM_LD(1, 9, 40); \
    TM_LD(1, 10, 46); \
    TM_LD(1, 11, 44); \
    prod = prod + ((YO(20) * YO(9)) * RCT(0, 0)); \
    loss = loss + (YO(27) * RCT(0, 1)); \
    prod = prod + ((YO(10) * YO(8)) * RCT(0, 2)); \
    loss = loss + (YO(27) * RCT(0, 3)); \
    prod = prod + ((YO(11) * YO(6)) * RCT(0, 4)); \
    loss = loss + (YO(28) * RCT(0, 5)); \
    prod = prod + ((YO(28) * YO(6)) * RCS(13)); \
    loss = loss + (YO(29) * RCS(12)); \
    prod = prod + (((YO(11) * YO(8)) * YO(4)) * RCS(27)); \
    loss = loss + (YO(23) * RCS(26)); \
    prod = prod + ((YO(23) * YO(6)) * RCS(32)); \
    loss = loss + (YO(31) * RCS(33)); \
    prod = prod + ((YO(34) * YO(6)) * RCS(61)); \
    loss = loss + (YO(31) * RCS(60)); \
    prod = prod + ((YO(31) * YO(6)) * RCS(105)); \
    loss = loss + (YO(35) * RCS(104)); \
    prod = prod + ((YO(31) * YO(6)) * RCS(115)); \
    loss = loss + (YO(32) * RCS(114)); \
    prod = prod + ((YO(37) * YO(6)) * RCS(136)); \
    loss = loss + (YO(36) * RCS(137)); \
    prod = prod + ((YO(25) * YO(10)) * RCS(141)); \
    loss = loss + (YO(37) * RCS(140)); \
    prod = prod + ((YO(36) * YO(6)) * RCS(147)); \
    loss = loss + (YO(38) * RCS(146)); \
    prod = prod + (((YO(13) * YO(10)) * YO(8)) * RCS(159)); \
    loss = loss + (YO(36) * RCS(158)); \
    prod = prod + ((YO(38) * YO(6)) * RCS(170)); \
    loss = loss + (YO(39) * RCS(171)); \
    prod = prod + ((YO(41) * YO(6)) * RCS(183)); \
    loss = loss + (YO(40) * RCS(182)); \
    prod = prod + ((YO(42) * YO(6)) * RCS(185)); \
    loss = loss + (YO(40) * RCS(184)); \
    prod = prod + ((YO(39) * YO(6)) * RCS(207)); \
    loss = loss + (YO(41) * RCS(206)); \
    prod = prod + ((YO(39) * YO(6)) * RCS(213)); \
    loss = loss + (YO(42) * RCS(212)); \
    prod = prod + (((YO(21) * YO(38)) * YO(6)) * RCS(237)); \
    loss = loss + (YO(45) * RCS(236)); \
    prod = prod + (((YO(22) * YO(36)) * YO(6)) * RCS(239)); \
    loss = loss + (YO(45) * RCS(238)); \
    loss = loss + (0.5 * SOUR(2)); \
    rhs1 = rho * Y0S(1) + dt * WM(1) * (prod + extra); \
    rhs2 = -(dt * WM(1) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(1) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(1) - fnew); \
    UC_UPDATE_TAIL(1); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 3); \
    prod = ((YO(4) * YO(3)) * RCT(0, 6)); \
    extra = 0.0; \
    loss = (YN(1) * RCT(0, 7)); \
    prod = prod + (YN(0) * (YO(3) * RCT(0, 8))); \
    loss = loss + (YO(4) * RCT(0, 9)); \
    prod = prod + (YN(0) * (YO(4) * RCT(0, 10))); \
    loss = loss + (YO(5) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 50); \
    TM_LD(0, 1, 48); \
    TM_LD(0, 2, 70); \
    TM_LD(0, 3, 68); \
    TM_LD(0, 4, 74); \
    TM_LD(0, 5, 72); \
    TM_LD(0, 6, 84); \
    TM_LD(0, 7, 86); \
    TM_LD(0, 8, 96); \
    TM_LD(0, 9, 98); \
    TM_LD(0, 10, 102); \
    TM_LD(0, 11, 100); \
    prod = prod + (YN(0) * RCT(1, 0)); \
    loss = loss + (YO(2) * RCT(1, 1)); \
    prod = prod + (YN(0) * RCT(1, 0)); \
    loss = loss + (YO(2) * RCT(1, 1)); \
    prod = prod + (YO(5) * RCT(1, 2)); \
    loss = loss + (YO(4) * RCT(1, 3)); \
    prod = prod + (YO(4) * RCT(1, 4)); \
    loss = loss + (YO(3) * RCT(1, 5)); \
    prod = prod + (YO(6) * RCT(1, 6)); \
    loss = loss + (YN(1) * RCT(1, 7)); \
    prod = prod + ((YO(4) * YO(4)) * RCT(1, 8)); \
    loss = loss + (YO(6) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YN(0) * RCT(1, 10))); \
    loss = loss + (YO(6) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 108); \
    TM_LD(1, 1, 110); \
    TM_LD(1, 2, 126); \
    TM_LD(1, 3, 124); \
    TM_LD(1, 4, 130); \
    TM_LD(1, 5, 128); \
    TM_LD(1, 6, 150); \
    TM_LD(1, 7, 148); \
    TM_LD(1, 8, 170); \
    TM_LD(1, 9, 168); \
    TM_LD(1, 10, 174); \
    TM_LD(1, 11, 172); \
    prod = prod + ((YO(5) * YO(3)) * RCT(0, 0)); \
    loss = loss + (YO(6) * RCT(0, 1)); \
    prod = prod + (YN(0) * (YO(6) * RCT(0, 2))); \
    loss = loss + (YO(7) * RCT(0, 3)); \
    prod = prod + ((YO(5) * YO(4)) * RCT(0, 4)); \
    loss = loss + (YO(7) * RCT(0, 5)); \
    prod = prod + ((YO(8) * YO(4)) * RCT(0, 6)); \
    loss = loss + (YO(9) * RCT(0, 7)); \
    prod = prod + (YO(10) * RCT(0, 8)); \
    loss = loss + (YO(8) * RCT(0, 9)); \
    prod = prod + (YN(0) * (YO(8) * RCT(0, 10))); \
    loss = loss + (YO(10) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 180); \
    TM_LD(0, 1, 182); \
    TM_LD(0, 2, 184); \
    TM_LD(0, 3, 186); \
    TM_LD(0, 4, 204); \
    TM_LD(0, 5, 206); \
    TM_LD(0, 6, 210); \
    TM_LD(0, 7, 208); \
    TM_LD(0, 8, 216); \
    TM_LD(0, 9, 218); \
    TM_LD(0, 10, 220); \
    TM_LD(0, 11, 222); \
    prod = prod + ((YO(10) * YO(3)) * RCT(1, 0)); \
    loss = loss + (YO(9) * RCT(1, 1)); \
    prod = prod + (YO(11) * RCT(1, 2)); \
    loss = loss + (YO(10) * RCT(1, 3)); \
    prod = prod + (YN(0) * (YO(10) * RCT(1, 4))); \
    loss = loss + (YO(11) * RCT(1, 5)); \
    prod = prod + (YN(0) * (YO(13) * RCT(1, 6))); \
    loss = loss + (YO(12) * RCT(1, 7)); \
    prod = prod + (YN(0) * (YO(14) * RCT(1, 8))); \
    loss = loss + (YO(13) * RCT(1, 9)); \
    prod = prod + (YN(0) * (YO(15) * RCT(1, 10))); \
    loss = loss + (YO(13) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 234); \
    TM_LD(1, 1, 232); \
    TM_LD(1, 2, 236); \
    TM_LD(1, 3, 238); \
    TM_LD(1, 4, 244); \
    TM_LD(1, 5, 246); \
    TM_LD(1, 6, 256); \
    TM_LD(1, 7, 258); \
    TM_LD(1, 8, 260); \
    TM_LD(1, 9, 262); \
    TM_LD(1, 10, 264); \
    TM_LD(1, 11, 266); \
    prod = prod + ((YO(13) * YO(3)) * RCT(0, 0)); \
    loss = loss + (YO(11) * RCT(0, 1)); \
    prod = prod + ((YO(13) * YO(14)) * RCT(0, 2)); \
    loss = loss + (YO(16) * RCT(0, 3)); \
    prod = prod + ((YO(13) * YO(13)) * RCT(0, 4)); \
    loss = loss + (YO(18) * RCT(0, 5)); \
    prod = prod + (YO(12) * RCT(0, 6)); \
    loss = loss + (YO(13) * RCT(0, 7)); \
    prod = prod + ((YO(15) * YO(4)) * RCT(0, 8)); \
    loss = loss + (YO(11) * RCT(0, 9)); \
    prod = prod + (YN(1) * (YO(15) * RCT(0, 10))); \
    loss = loss + ((YO(8) * YO(4)) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 272); \
    TM_LD(0, 1, 274); \
    TM_LD(0, 2, 282); \
    TM_LD(0, 3, 280); \
    TM_LD(0, 4, 286); \
    TM_LD(0, 5, 284); \
    TM_LD(0, 6, 300); \
    TM_LD(0, 7, 302); \
    TM_LD(0, 8, 306); \
    TM_LD(0, 9, 304); \
    TM_LD(0, 10, 320); \
    TM_LD(0, 11, 322); \
    prod = prod + (YN(0) * (YO(20) * RCT(1, 0))); \
    loss = loss + (YO(14) * RCT(1, 1)); \
    prod = prod + ((YO(14) * YO(4)) * RCT(1, 2)); \
    loss = loss + (YO(11) * RCT(1, 3)); \
    prod = prod + ((YO(14) * YO(3)) * RCT(1, 4)); \
    loss = loss + ((YO(8) * YO(2)) * RCT(1, 5)); \
    prod = prod + ((YO(14) * YO(3)) * RCT(1, 4)); \
    loss = loss + ((YO(8) * YO(2)) * RCT(1, 5)); \
    prod = prod + (YN(1) * (YO(14) * RCT(1, 6))); \
    loss = loss + ((YO(8) * YO(4)) * RCT(1, 7)); \
    prod = prod + ((YO(14) * YO(14)) * RCT(1, 8)); \
    loss = loss + ((YO(21) * YO(2)) * RCT(1, 9)); \
    prod = prod + ((YO(14) * YO(14)) * RCT(1, 8)); \
    loss = loss + ((YO(21) * YO(2)) * RCT(1, 9)); \
    prod = prod + ((YO(20) * YO(3)) * RCT(1, 10)); \
    loss = loss + (YO(8) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 330); \
    TM_LD(1, 1, 328); \
    TM_LD(1, 2, 344); \
    TM_LD(1, 3, 346); \
    TM_LD(1, 4, 350); \
    TM_LD(1, 5, 348); \
    TM_LD(1, 6, 360); \
    TM_LD(1, 7, 362); \
    TM_LD(1, 8, 380); \
    TM_LD(1, 9, 382); \
    TM_LD(1, 10, 390); \
    TM_LD(1, 11, 388); \
    prod = prod + ((YO(20) * YO(5)) * RCT(0, 0)); \
    loss = loss + (YO(11) * RCT(0, 1)); \
    prod = prod + (YN(0) * (YO(11) * RCT(0, 2))); \
    loss = loss + (YO(17) * RCT(0, 3)); \
    prod = prod + ((YO(15) * YO(5)) * RCT(0, 4)); \
    loss = loss + (YO(17) * RCT(0, 5)); \
    prod = prod + (YO(17) * RCT(0, 6)); \
    loss = loss + (YO(11) * RCT(0, 7)); \
    prod = prod + (YN(0) * (YO(18) * RCT(0, 8))); \
    loss = loss + (YO(19) * RCT(0, 9)); \
    prod = prod + (YO(19) * RCT(0, 10)); \
    loss = loss + (YO(18) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 392); \
    TM_LD(0, 1, 394); \
    TM_LD(0, 2, 408); \
    TM_LD(0, 3, 410); \
    TM_LD(0, 4, 420); \
    TM_LD(0, 5, 422); \
    TM_LD(0, 6, 430); \
    TM_LD(0, 7, 428); \
    TM_LD(0, 8, 446); \
    TM_LD(0, 9, 444); \
    TM_LD(0, 10, 448); \
    TM_LD(0, 11, 450); \
    prod = prod + (YN(0) * (YO(16) * RCT(1, 0))); \
    loss = loss + (YO(18) * RCT(1, 1)); \
    prod = prod + (YO(18) * RCT(1, 2)); \
    loss = loss + (YO(16) * RCT(1, 3)); \
    prod = prod + (YN(0) * (YO(22) * RCT(1, 4))); \
    loss = loss + (YO(16) * RCT(1, 5)); \
    prod = prod + ((YO(16) * YO(3)) * RCT(1, 6)); \
    loss = loss + (YO(23) * RCT(1, 7)); \
    prod = prod + (YO(16) * RCT(1, 8)); \
    loss = loss + (YO(22) * RCT(1, 9)); \
    prod = prod + (YN(0) * (YO(21) * RCT(1, 10))); \
    loss = loss + (YO(22) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 452); \
    TM_LD(1, 1, 454); \
    TM_LD(1, 2, 460); \
    TM_LD(1, 3, 462); \
    TM_LD(1, 4, 464); \
    TM_LD(1, 5, 466); \
    TM_LD(1, 6, 486); \
    TM_LD(1, 7, 484); \
    TM_LD(1, 8, 490); \
    TM_LD(1, 9, 488); \
    TM_LD(1, 10, 500); \
    TM_LD(1, 11, 502); \
    prod = prod + (YO(22) * RCT(0, 0)); \
    loss = loss + (YO(21) * RCT(0, 1)); \
    prod = prod + ((YO(21) * YO(3)) * RCT(0, 2)); \
    loss = loss + (YO(26) * RCT(0, 3)); \
    prod = prod + ((YO(21) * YO(4)) * RCT(0, 4)); \
    loss = loss + (YO(25) * RCT(0, 5)); \
    prod = prod + ((YO(13) * YO(8)) * RCT(0, 6)); \
    loss = loss + (YO(25) * RCT(0, 7)); \
    prod = prod + ((YO(15) * YO(8)) * RCT(0, 8)); \
    loss = loss + (YO(26) * RCT(0, 9)); \
    prod = prod + ((YO(26) * YO(4)) * RCT(0, 10)); \
    loss = loss + ((YO(10) * YO(8)) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 0); \
    TM_LD(0, 1, 2); \
    TM_LD(0, 2, 6); \
    TM_LD(0, 3, 4); \
    TM_LD(0, 4, 14); \
    TM_LD(0, 5, 12); \
    TM_LD(0, 6, 26); \
    TM_LD(0, 7, 24); \
    TM_LD(0, 8, 30); \
    TM_LD(0, 9, 28); \
    TM_LD(0, 10, 34); \
    TM_LD(0, 11, 32); \
    prod = prod + ((YO(26) * YO(3)) * RCT(1, 0)); \
    loss = loss + ((YO(8) * YO(8)) * RCT(1, 1)); \
    prod = prod + (YN(1) * (YO(26) * RCT(1, 2))); \
    loss = loss + ((YO(9) * YO(8)) * RCT(1, 3)); \
    prod = prod + ((YO(27) * YO(4)) * RCT(1, 4)); \
    loss = loss + (YO(26) * RCT(1, 5)); \
    prod = prod + (YN(0) * (YO(11) * RCT(1, 6))); \
    loss = loss + (YO(28) * RCT(1, 7)); \
    prod = prod + ((YO(13) * YO(4)) * RCT(1, 8)); \
    loss = loss + (YO(28) * RCT(1, 9)); \
    prod = prod + (YO(28) * RCT(1, 10)); \
    loss = loss + (YO(11) * RCT(1, 11)); \
    prod = prod + (YN(0) * (YO(28) * RCS(5))); \
    loss = loss + (YO(29) * RCS(4)); \
    prod = prod + (YN(0) * (YO(17) * RCS(7))); \
    loss = loss + (YO(29) * RCS(6)); \
    prod = prod + (YO(23) * RCS(16)); \
    loss = loss + (YO(25) * RCS(17)); \
    prod = prod + ((YO(13) * YO(10)) * RCS(19)); \
    loss = loss + (YO(23) * RCS(18)); \
    prod = prod + (YN(0) * (YO(25) * RCS(21))); \
    loss = loss + (YO(23) * RCS(20)); \
    prod = prod + ((YO(23) * YO(13)) * RCS(28)); \
    loss = loss + ((YO(18) * YO(8)) * RCS(29)); \
    prod = prod + (YN(0) * (YO(34) * RCS(49))); \
    loss = loss + (YO(31) * RCS(48)); \
    prod = prod + (YN(0) * (YO(23) * RCS(51))); \
    loss = loss + (YO(31) * RCS(50)); \
    prod = prod + (YN(0) * (YO(33) * RCS(73))); \
    loss = loss + (YO(30) * RCS(72)); \
    prod = prod + (YN(0) * (YO(32) * RCS(75))); \
    loss = loss + (YO(30) * RCS(74)); \
    prod = prod + (YN(0) * (YO(35) * RCS(77))); \
    loss = loss + (YO(30) * RCS(76)); \
    prod = prod + (YO(35) * RCS(100)); \
    loss = loss + (YO(31) * RCS(101)); \
    prod = prod + ((YO(13) * YO(28)) * RCS(109)); \
    loss = loss + (YO(35) * RCS(108)); \
    prod = prod + ((YO(16) * YO(5)) * RCS(111)); \
    loss = loss + (YO(35) * RCS(110)); \
    prod = prod + ((YO(16) * YO(5)) * RCS(119)); \
    loss = loss + (YO(32) * RCS(118)); \
    prod = prod + ((YO(13) * YO(28)) * RCS(121)); \
    loss = loss + (YO(32) * RCS(120)); \
    prod = prod + (YO(32) * RCS(126)); \
    loss = loss + (YO(31) * RCS(127)); \
    prod = prod + ((YO(13) * YO(21)) * RCS(130)); \
    loss = loss + (YO(36) * RCS(131)); \
    prod = prod + (YO(36) * RCS(135)); \
    loss = loss + (YO(37) * RCS(134)); \
    prod = prod + (YO(38) * RCS(143)); \
    loss = loss + (YO(36) * RCS(142)); \
    prod = prod + (YN(0) * (YO(36) * RCS(145))); \
    loss = loss + (YO(38) * RCS(144)); \
    prod = prod + ((YO(39) * YO(3)) * RCS(164)); \
    loss = loss + ((YO(25) * YO(13)) * RCS(165)); \
    prod = prod + (YN(0) * (YO(38) * RCS(167))); \
    loss = loss + (YO(39) * RCS(166)); \
    prod = prod + (YO(39) * RCS(169)); \
    loss = loss + (YO(38) * RCS(168)); \
    prod = prod + ((YO(16) * YO(13)) * RCS(177)); \
    loss = loss + (YO(39) * RCS(176)); \
    prod = prod + ((YO(13) * YO(22)) * RCS(178)); \
    loss = loss + (YO(38) * RCS(179)); \
    prod = prod + (YN(0) * (YO(41) * RCS(187))); \
    loss = loss + (YO(40) * RCS(186)); \
    prod = prod + (YN(0) * (YO(42) * RCS(189))); \
    loss = loss + (YO(40) * RCS(188)); \
    prod = prod + (YO(41) * RCS(205)); \
    loss = loss + (YO(39) * RCS(204)); \
    prod = prod + (YO(42) * RCS(211)); \
    loss = loss + (YO(39) * RCS(210)); \
    prod = prod + (YO(43) * RCS(214)); \
    loss = loss + ((YO(21) * YO(22)) * RCS(215)); \
    prod = prod + ((YO(22) * YO(16)) * RCS(221)); \
    loss = loss + (YO(43) * RCS(220)); \
    prod = prod + (YN(0) * ((YO(21) * YO(22)) * RCS(223))); \
    loss = loss + (YO(43) * RCS(222)); \
    prod = prod + ((YO(43) * YO(4)) * RCS(224)); \
    loss = loss + ((YO(44) * YO(38)) * RCS(225)); \
    prod = prod + 0.0; \
    loss = loss + (YO(46) * RCS(246)); \
    prod = prod + 0.0; \
    loss = loss + (YO(46) * RCS(248)); \
    prod = prod + 0.0; \
    loss = loss + (YO(46) * RCS(250)); \
    prod = prod + (YN(0) * ((YO(48) * YO(18)) * RCS(253))); \
    loss = loss + (YO(46) * RCS(252)); \
    prod = prod + (YN(0) * ((YO(39) * YO(22)) * RCS(269))); \
    loss = loss + (YO(48) * RCS(268)); \
    prod = prod + (((YO(16) * YO(16)) * YO(13)) * RCS(271)); \
    loss = loss + (YO(48) * RCS(270)); \
    prod = prod + ((YO(39) * YO(18)) * RCS(273)); \
    loss = loss + (YO(48) * RCS(272)); \
    prod = prod + (YN(0) * ((YO(16) * YO(38)) * RCS(275))); \
    loss = loss + (YO(48) * RCS(274)); \
    prod = prod + (YN(0) * ((YO(43) * YO(13)) * RCS(277))); \
    loss = loss + (YO(48) * RCS(276)); \
    prod = prod + ((YO(16) * YO(18)) * RCS(281)); \
    loss = loss + (YO(47) * RCS(280)); \
    prod = prod + ((YO(39) * YO(13)) * RCS(283)); \
    loss = loss + (YO(47) * RCS(282)); \
    prod = prod + (YN(0) * ((YO(22) * YO(16)) * RCS(285))); \
    loss = loss + (YO(47) * RCS(284)); \
    prod = prod + ((YO(47) * YO(4)) * RCS(286)); \
    loss = loss + ((YO(5) * YO(43)) * RCS(287)); \
    prod = prod + (SOUR(3) * YO(4)); \
    rhs1 = rho * Y0S(0) + dt * WM(2) * (prod + extra); \
    rhs2 = -(dt * WM(2) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(2) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(2) - fnew); \
    UC_UPDATE_TAIL(2); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 4); \
    TM_WAIT(0); \
    TM_LD(1, 0, 48); \
    TM_LD(1, 1, 50); \
    TM_LD(1, 2, 54); \
    TM_LD(1, 3, 52); \
    TM_LD(1, 4, 82); \
    TM_LD(1, 5, 80); \
    TM_LD(1, 6, 92); \
    TM_LD(1, 7, 94); \
    TM_LD(1, 8, 106); \
    TM_LD(1, 9, 104); \
    TM_LD(1, 10, 110); \
    TM_LD(1, 11, 108); \
    prod = (YN(2) * (YN(1) * RCT(0, 0))); \
    extra = 0.0; \
    loss = (YO(4) * RCT(0, 1)); \
    prod = prod + (YN(2) * (YO(4) * RCT(0, 2))); \
    loss = loss + (YN(0) * RCT(0, 3)); \
    prod = prod + ((YO(4) * YO(4)) * RCT(0, 4)); \
    loss = loss + (YO(5) * RCT(0, 5)); \
    prod = prod + (YN(1) * RCT(0, 6)); \
    loss = loss + (YO(3) * RCT(0, 7)); \
    prod = prod + (YN(1) * RCT(0, 6)); \
    loss = loss + (YO(3) * RCT(0, 7)); \
    prod = prod + (YO(4) * RCT(0, 8)); \
    loss = loss + (YN(2) * RCT(0, 9)); \
    prod = prod + (YO(6) * RCT(0, 10)); \
    loss = loss + (YO(4) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 134); \
    TM_LD(0, 1, 132); \
    TM_LD(0, 2, 158); \
    TM_LD(0, 3, 156); \
    TM_LD(0, 4, 182); \
    TM_LD(0, 5, 180); \
    TM_LD(0, 6, 196); \
    TM_LD(0, 7, 198); \
    TM_LD(0, 8, 246); \
    TM_LD(0, 9, 244); \
    TM_LD(0, 10, 250); \
    TM_LD(0, 11, 248); \
    prod = prod + (YN(2) * (YO(6) * RCT(1, 0))); \
    loss = loss + (YO(5) * RCT(1, 1)); \
    prod = prod + (YN(1) * (YO(4) * RCT(1, 2))); \
    loss = loss + (YO(6) * RCT(1, 3)); \
    prod = prod + ((YO(6) * YO(4)) * RCT(1, 4)); \
    loss = loss + (YO(7) * RCT(1, 5)); \
    prod = prod + (YN(1) * (YO(8) * RCT(1, 6))); \
    loss = loss + (YO(9) * RCT(1, 7)); \
    prod = prod + ((YO(8) * YO(4)) * RCT(1, 8)); \
    loss = loss + (YO(10) * RCT(1, 9)); \
    prod = prod + (YN(2) * (YO(9) * RCT(1, 10))); \
    loss = loss + (YO(10) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 266); \
    TM_LD(1, 1, 264); \
    TM_LD(1, 2, 268); \
    TM_LD(1, 3, 270); \
    TM_LD(1, 4, 294); \
    TM_LD(1, 5, 292); \
    TM_LD(1, 6, 310); \
    TM_LD(1, 7, 308); \
    TM_LD(1, 8, 334); \
    TM_LD(1, 9, 332); \
    TM_LD(1, 10, 338); \
    TM_LD(1, 11, 336); \
    prod = prod + ((YO(10) * YO(4)) * RCT(0, 0)); \
    loss = loss + (YO(11) * RCT(0, 1)); \
    prod = prod + ((YO(13) * YO(4)) * RCT(0, 2)); \
    loss = loss + (YO(12) * RCT(0, 3)); \
    prod = prod + (YN(2) * (YO(11) * RCT(0, 4))); \
    loss = loss + (YO(13) * RCT(0, 5)); \
    prod = prod + (YN(1) * (YO(13) * RCT(0, 6))); \
    loss = loss + (YO(17) * RCT(0, 7)); \
    prod = prod + (YN(2) * ((YO(8) * YOS(0)) * RCT(0, 8))); \
    loss = loss + (YO(14) * RCT(0, 9)); \
    prod = prod + (YN(0) * (YO(8) * RCT(0, 10))); \
    loss = loss + (YO(14) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 358); \
    TM_LD(0, 1, 356); \
    TM_LD(0, 2, 362); \
    TM_LD(0, 3, 360); \
    TM_LD(0, 4, 400); \
    TM_LD(0, 5, 402); \
    TM_LD(0, 6, 410); \
    TM_LD(0, 7, 408); \
    TM_LD(0, 8, 414); \
    TM_LD(0, 9, 412); \
    TM_LD(0, 10, 434); \
    TM_LD(0, 11, 432); \
    prod = prod + (YN(2) * (YO(8) * RCT(1, 0))); \
    loss = loss + (YO(20) * RCT(1, 1)); \
    prod = prod + (YN(1) * (YO(20) * RCT(1, 2))); \
    loss = loss + (YO(10) * RCT(1, 3)); \
    prod = prod + ((YO(4) * YO(11)) * RCT(1, 4)); \
    loss = loss + (YO(17) * RCT(1, 5)); \
    prod = prod + ((YO(18) * YO(4)) * RCT(1, 6)); \
    loss = loss + (YO(19) * RCT(1, 7)); \
    prod = prod + ((YO(16) * YO(4)) * RCT(1, 8)); \
    loss = loss + (YO(18) * RCT(1, 9)); \
    prod = prod + ((YO(13) * YO(11)) * RCT(1, 10)); \
    loss = loss + (YO(18) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 438); \
    TM_LD(1, 1, 436); \
    TM_LD(1, 2, 454); \
    TM_LD(1, 3, 452); \
    TM_LD(1, 4, 470); \
    TM_LD(1, 5, 468); \
    TM_LD(1, 6, 472); \
    TM_LD(1, 7, 474); \
    TM_LD(1, 8, 0); \
    TM_LD(1, 9, 2); \
    TM_LD(1, 10, 4); \
    TM_LD(1, 11, 6); \
    prod = prod + ((YO(13) * YO(10)) * RCT(0, 0)); \
    loss = loss + (YO(16) * RCT(0, 1)); \
    prod = prod + (YN(2) * (YO(23) * RCT(0, 2))); \
    loss = loss + (YO(16) * RCT(0, 3)); \
    prod = prod + (YN(1) * (YO(22) * RCT(0, 4))); \
    loss = loss + (YO(23) * RCT(0, 5)); \
    prod = prod + (YN(2) * (YO(26) * RCT(0, 6))); \
    loss = loss + (YO(21) * RCT(0, 7)); \
    prod = prod + ((YO(14) * YO(8)) * RCT(0, 8)); \
    loss = loss + (YO(21) * RCT(0, 9)); \
    prod = prod + ((YO(14) * YO(9)) * RCT(0, 10)); \
    loss = loss + (YO(25) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 10); \
    TM_LD(0, 1, 8); \
    TM_LD(0, 2, 12); \
    TM_LD(0, 3, 14); \
    TM_LD(0, 4, 22); \
    TM_LD(0, 5, 20); \
    TM_LD(0, 6, 28); \
    TM_LD(0, 7, 30); \
    TM_LD(0, 8, 34); \
    TM_LD(0, 9, 32); \
    TM_LD(0, 10, 40); \
    TM_LD(0, 11, 42); \
    prod = prod + ((YO(26) * YO(4)) * RCT(1, 0)); \
    loss = loss + (YO(25) * RCT(1, 1)); \
    prod = prod + (YN(2) * ((YO(8) * YO(8)) * RCT(1, 2))); \
    loss = loss + (YO(26) * RCT(1, 3)); \
    prod = prod + ((YO(8) * YO(20)) * RCT(1, 4)); \
    loss = loss + (YO(27) * RCT(1, 5)); \
    prod = prod + (YN(1) * (YO(27) * RCT(1, 6))); \
    loss = loss + (YO(26) * RCT(1, 7)); \
    prod = prod + ((YO(28) * YO(4)) * RCS(9)); \
    loss = loss + (YO(29) * RCS(8)); \
    prod = prod + ((YO(11) * YO(10)) * RCS(23)); \
    loss = loss + (YO(23) * RCS(22)); \
    prod = prod + ((YO(34) * YO(4)) * RCS(45)); \
    loss = loss + (YO(31) * RCS(44)); \
    prod = prod + ((YO(23) * YO(4)) * RCS(47)); \
    loss = loss + (YO(31) * RCS(46)); \
    prod = prod + ((YO(33) * YO(4)) * RCS(79)); \
    loss = loss + (YO(30) * RCS(78)); \
    prod = prod + ((YO(32) * YO(4)) * RCS(81)); \
    loss = loss + (YO(30) * RCS(80)); \
    prod = prod + ((YO(35) * YO(4)) * RCS(83)); \
    loss = loss + (YO(30) * RCS(82)); \
    prod = prod + ((YO(31) * YO(4)) * RCS(117)); \
    loss = loss + (YO(32) * RCS(116)); \
    prod = prod + ((YO(16) * YO(8)) * RCS(129)); \
    loss = loss + (YO(36) * RCS(128)); \
    prod = prod + ((YO(26) * YO(13)) * RCS(133)); \
    loss = loss + (YO(36) * RCS(132)); \
    prod = prod + ((YO(18) * YO(10)) * RCS(161)); \
    loss = loss + (YO(39) * RCS(160)); \
    prod = prod + (YN(2) * ((YO(25) * YO(13)) * RCS(165))); \
    loss = loss + (YO(39) * RCS(164)); \
    prod = prod + ((YO(41) * YO(4)) * RCS(191)); \
    loss = loss + (YO(40) * RCS(190)); \
    prod = prod + ((YO(42) * YO(4)) * RCS(193)); \
    loss = loss + (YO(40) * RCS(192)); \
    loss = loss + SOUR(4); \
    rhs1 = rho * Y0S(1) + dt * WM(3) * (prod + extra); \
    rhs2 = -(dt * WM(3) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(3) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(3) - fnew); \
    UC_UPDATE_TAIL(3); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 5); \
    prod = (YN(2) * (YN(1) * RCT(1, 8))); \
    extra = 0.0; \
    loss = (YN(3) * RCT(1, 9)); \
    prod = prod + (YN(3) * (YN(0) * RCT(1, 10))); \
    loss = loss + (YN(2) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 52); \
    TM_LD(1, 1, 54); \
    TM_LD(1, 2, 58); \
    TM_LD(1, 3, 56); \
    TM_LD(1, 4, 62); \
    TM_LD(1, 5, 60); \
    TM_LD(1, 6, 72); \
    TM_LD(1, 7, 74); \
    TM_LD(1, 8, 78); \
    TM_LD(1, 9, 76); \
    TM_LD(1, 10, 80); \
    TM_LD(1, 11, 82); \
    prod = prod + (YN(2) * (YO(5) * RCT(0, 0))); \
    loss = loss + (YN(0) * RCT(0, 1)); \
    prod = prod + (YN(3) * (YO(5) * RCT(0, 2))); \
    loss = loss + (YO(4) * RCT(0, 3)); \
    prod = prod + (YN(3) * (YO(5) * RCT(0, 2))); \
    loss = loss + (YO(4) * RCT(0, 3)); \
    prod = prod + (YO(5) * RCT(0, 4)); \
    loss = loss + (YN(2) * RCT(0, 5)); \
    prod = prod + (YN(3) * (YN(2) * RCT(0, 6))); \
    loss = loss + RCT(0, 7); \
    prod = prod + (YO(6) * RCT(0, 8)); \
    loss = loss + (YN(3) * RCT(0, 9)); \
    prod = prod + (YN(2) * (YO(6) * RCT(0, 10))); \
    loss = loss + (YO(4) * RCT(0, 11)); \
    prod = prod + (YN(2) * (YO(6) * RCT(0, 10))); \
    loss = loss + (YO(4) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 86); \
    TM_LD(0, 1, 84); \
    TM_LD(0, 2, 88); \
    TM_LD(0, 3, 90); \
    TM_LD(0, 4, 104); \
    TM_LD(0, 5, 106); \
    TM_LD(0, 6, 114); \
    TM_LD(0, 7, 112); \
    TM_LD(0, 8, 132); \
    TM_LD(0, 9, 134); \
    TM_LD(0, 10, 138); \
    TM_LD(0, 11, 136); \
    prod = prod + (YN(3) * (YO(6) * RCT(1, 0))); \
    loss = loss + (YN(1) * RCT(1, 1)); \
    prod = prod + (YN(1) * (YO(5) * RCT(1, 2))); \
    loss = loss + (YO(6) * RCT(1, 3)); \
    prod = prod + (YO(7) * RCT(1, 4)); \
    loss = loss + (YO(4) * RCT(1, 5)); \
    prod = prod + (YO(7) * RCT(1, 4)); \
    loss = loss + (YO(4) * RCT(1, 5)); \
    prod = prod + (YN(2) * (YO(7) * RCT(1, 6))); \
    loss = loss + (YO(5) * RCT(1, 7)); \
    prod = prod + ((YO(5) * YO(6)) * RCT(1, 8)); \
    loss = loss + (YO(7) * RCT(1, 9)); \
    prod = prod + (YN(3) * (YO(7) * RCT(1, 10))); \
    loss = loss + (YO(6) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 154); \
    TM_LD(1, 1, 152); \
    TM_LD(1, 2, 156); \
    TM_LD(1, 3, 158); \
    TM_LD(1, 4, 178); \
    TM_LD(1, 5, 176); \
    TM_LD(1, 6, 188); \
    TM_LD(1, 7, 190); \
    TM_LD(1, 8, 192); \
    TM_LD(1, 9, 194); \
    TM_LD(1, 10, 218); \
    TM_LD(1, 11, 216); \
    prod = prod + (YN(2) * (YO(9) * RCT(0, 0))); \
    loss = loss + (YO(8) * RCT(0, 1)); \
    prod = prod + ((YO(8) * YO(6)) * RCT(0, 2)); \
    loss = loss + (YO(9) * RCT(0, 3)); \
    prod = prod + (YN(3) * (YO(10) * RCT(0, 4))); \
    loss = loss + (YO(8) * RCT(0, 5)); \
    prod = prod + ((YO(8) * YO(5)) * RCT(0, 6)); \
    loss = loss + (YO(10) * RCT(0, 7)); \
    prod = prod + (YN(3) * (YO(11) * RCT(0, 8))); \
    loss = loss + (YO(10) * RCT(0, 9)); \
    prod = prod + ((YO(10) * YO(5)) * RCT(0, 10)); \
    loss = loss + (YO(11) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 220); \
    TM_LD(0, 1, 222); \
    TM_LD(0, 2, 238); \
    TM_LD(0, 3, 236); \
    TM_LD(0, 4, 242); \
    TM_LD(0, 5, 240); \
    TM_LD(0, 6, 256); \
    TM_LD(0, 7, 258); \
    TM_LD(0, 8, 290); \
    TM_LD(0, 9, 288); \
    TM_LD(0, 10, 292); \
    TM_LD(0, 11, 294); \
    prod = prod + ((YO(5) * YO(13)) * RCT(1, 0)); \
    loss = loss + (YO(12) * RCT(1, 1)); \
    prod = prod + (YN(3) * (YO(12) * RCT(1, 2))); \
    loss = loss + (YO(13) * RCT(1, 3)); \
    prod = prod + ((YO(15) * YO(5)) * RCT(1, 4)); \
    loss = loss + (YO(13) * RCT(1, 5)); \
    prod = prod + ((YO(13) * YO(6)) * RCT(1, 6)); \
    loss = loss + (YO(17) * RCT(1, 7)); \
    prod = prod + (YN(1) * (YO(13) * RCT(1, 8))); \
    loss = loss + (YO(11) * RCT(1, 9)); \
    prod = prod + (YN(2) * (YO(11) * RCT(1, 10))); \
    loss = loss + (YO(15) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 308); \
    TM_LD(1, 1, 310); \
    TM_LD(1, 2, 314); \
    TM_LD(1, 3, 312); \
    TM_LD(1, 4, 332); \
    TM_LD(1, 5, 334); \
    TM_LD(1, 6, 354); \
    TM_LD(1, 7, 352); \
    TM_LD(1, 8, 372); \
    TM_LD(1, 9, 374); \
    TM_LD(1, 10, 422); \
    TM_LD(1, 11, 420); \
    prod = prod + (YN(1) * (YO(15) * RCT(0, 0))); \
    loss = loss + ((YO(8) * YN(2)) * RCT(0, 1)); \
    prod = prod + (YN(2) * (YO(11) * RCT(0, 2))); \
    loss = loss + (YO(14) * RCT(0, 3)); \
    prod = prod + ((YO(20) * YO(5)) * RCT(0, 4)); \
    loss = loss + (YO(14) * RCT(0, 5)); \
    prod = prod + (YN(1) * (YO(14) * RCT(0, 6))); \
    loss = loss + ((YO(8) * YN(2)) * RCT(0, 7)); \
    prod = prod + ((YO(11) * YO(5)) * RCT(0, 8)); \
    loss = loss + (YO(17) * RCT(0, 9)); \
    prod = prod + (YN(3) * (YO(17) * RCT(0, 10))); \
    loss = loss + (YO(11) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 426); \
    TM_LD(0, 1, 424); \
    TM_LD(0, 2, 436); \
    TM_LD(0, 3, 438); \
    TM_LD(0, 4, 450); \
    TM_LD(0, 5, 448); \
    TM_LD(0, 6, 456); \
    TM_LD(0, 7, 458); \
    TM_LD(0, 8, 466); \
    TM_LD(0, 9, 464); \
    TM_LD(0, 10, 488); \
    TM_LD(0, 11, 490); \
    prod = prod + (YN(3) * (YO(19) * RCT(1, 0))); \
    loss = loss + (YO(18) * RCT(1, 1)); \
    prod = prod + ((YO(18) * YO(5)) * RCT(1, 2)); \
    loss = loss + (YO(19) * RCT(1, 3)); \
    prod = prod + (YN(3) * (YO(18) * RCT(1, 4))); \
    loss = loss + (YO(16) * RCT(1, 5)); \
    prod = prod + ((YO(22) * YO(5)) * RCT(1, 6)); \
    loss = loss + (YO(16) * RCT(1, 7)); \
    prod = prod + ((YO(16) * YO(6)) * RCT(1, 8)); \
    loss = loss + (YO(24) * RCT(1, 9)); \
    prod = prod + (YN(2) * (YO(25) * RCT(1, 10))); \
    loss = loss + (YO(21) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 494); \
    TM_LD(1, 1, 492); \
    TM_LD(1, 2, 510); \
    TM_LD(1, 3, 508); \
    TM_LD(1, 4, 8); \
    TM_LD(1, 5, 10); \
    TM_LD(1, 6, 14); \
    TM_LD(1, 7, 12); \
    TM_LD(1, 8, 20); \
    TM_LD(1, 9, 22); \
    TM_LD(1, 10, 48); \
    TM_LD(1, 11, 50); \
    prod = prod + ((YO(27) * YO(5)) * RCT(0, 0)); \
    loss = loss + (YO(21) * RCT(0, 1)); \
    prod = prod + (YN(3) * (YO(25) * RCT(0, 2))); \
    loss = loss + (YO(26) * RCT(0, 3)); \
    prod = prod + (YN(2) * ((YO(10) * YO(8)) * RCT(0, 4))); \
    loss = loss + (YO(26) * RCT(0, 5)); \
    prod = prod + (YN(1) * (YO(26) * RCT(0, 6))); \
    loss = loss + ((YO(8) * YO(8)) * RCT(0, 7)); \
    prod = prod + (YN(2) * (YO(26) * RCT(0, 8))); \
    loss = loss + (YO(27) * RCT(0, 9)); \
    prod = prod + (YN(2) * (YO(28) * RCT(0, 10))); \
    loss = loss + (YO(13) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 56); \
    TM_LD(0, 1, 58); \
    TM_LD(0, 2, 72); \
    TM_LD(0, 3, 74); \
    TM_LD(0, 4, 76); \
    TM_LD(0, 5, 78); \
    TM_LD(0, 6, 112); \
    TM_LD(0, 7, 114); \
    TM_LD(0, 8, 136); \
    TM_LD(0, 9, 138); \
    TM_LD(0, 10, 152); \
    TM_LD(0, 11, 154); \
    prod = prod + ((YO(11) * YO(5)) * RCT(1, 0)); \
    loss = loss + (YO(28) * RCT(1, 1)); \
    prod = prod + ((YO(28) * YO(8)) * RCT(1, 2)); \
    loss = loss + (YO(25) * RCT(1, 3)); \
    prod = prod + ((YO(28) * YO(5)) * RCS(1)); \
    loss = loss + (YO(29) * RCS(0)); \
    prod = prod + ((YO(17) * YO(5)) * RCS(3)); \
    loss = loss + (YO(29) * RCS(2)); \
    prod = prod + (YN(3) * (YO(29) * RCS(8))); \
    loss = loss + (YO(28) * RCS(9)); \
    prod = prod + (YO(29) * RCS(14)); \
    loss = loss + (YO(13) * RCS(15)); \
    prod = prod + ((YO(25) * YO(5)) * RCS(25)); \
    loss = loss + (YO(23) * RCS(24)); \
    prod = prod + (YN(1) * (YO(23) * RCS(26))); \
    loss = loss + ((YO(11) * YO(8)) * RCS(27)); \
    prod = prod + ((YO(23) * YO(6)) * RCS(30)); \
    loss = loss + ((YO(11) * YO(10)) * RCS(31)); \
    prod = prod + ((YO(34) * YO(5)) * RCS(41)); \
    loss = loss + (YO(31) * RCS(40)); \
    prod = prod + ((YO(23) * YO(5)) * RCS(43)); \
    loss = loss + (YO(31) * RCS(42)); \
    prod = prod + (YN(3) * (YO(31) * RCS(44))); \
    loss = loss + (YO(34) * RCS(45)); \
    prod = prod + (YN(3) * (YO(31) * RCS(46))); \
    loss = loss + (YO(23) * RCS(47)); \
    prod = prod + ((YO(33) * YO(5)) * RCS(67)); \
    loss = loss + (YO(30) * RCS(66)); \
    prod = prod + ((YO(32) * YO(5)) * RCS(69)); \
    loss = loss + (YO(30) * RCS(68)); \
    prod = prod + ((YO(35) * YO(5)) * RCS(71)); \
    loss = loss + (YO(30) * RCS(70)); \
    prod = prod + (YN(3) * (YO(30) * RCS(78))); \
    loss = loss + (YO(33) * RCS(79)); \
    prod = prod + (YN(3) * (YO(30) * RCS(80))); \
    loss = loss + (YO(32) * RCS(81)); \
    prod = prod + (YN(3) * (YO(30) * RCS(82))); \
    loss = loss + (YO(35) * RCS(83)); \
    prod = prod + (YO(33) * RCS(97)); \
    loss = loss + (YO(16) * RCS(96)); \
    prod = prod + ((YO(18) * YO(6)) * RCS(98)); \
    loss = loss + (YO(35) * RCS(99)); \
    prod = prod + ((YO(31) * YO(5)) * RCS(113)); \
    loss = loss + (YO(35) * RCS(112)); \
    prod = prod + (YN(3) * (YO(32) * RCS(116))); \
    loss = loss + (YO(31) * RCS(117)); \
    prod = prod + ((YO(32) * YO(6)) * RCS(122)); \
    loss = loss + ((YO(31) * YO(4)) * RCS(123)); \
    prod = prod + ((YO(32) * YO(6)) * RCS(122)); \
    loss = loss + ((YO(31) * YO(4)) * RCS(123)); \
    prod = prod + ((YO(31) * YO(5)) * RCS(125)); \
    loss = loss + (YO(32) * RCS(124)); \
    prod = prod + ((YO(37) * YO(5)) * RCS(139)); \
    loss = loss + (YO(36) * RCS(138)); \
    prod = prod + ((YO(36) * YO(5)) * RCS(153)); \
    loss = loss + (YO(38) * RCS(152)); \
    prod = prod + ((YO(37) * YO(6)) * RCS(156)); \
    loss = loss + ((YO(8) * YO(22)) * RCS(157)); \
    prod = prod + ((YO(38) * YO(5)) * RCS(163)); \
    loss = loss + (YO(39) * RCS(162)); \
    prod = prod + ((YO(38) * YO(6)) * RCS(172)); \
    loss = loss + ((YO(22) * YO(11)) * RCS(173)); \
    prod = prod + (YN(3) * (YO(40) * RCS(190))); \
    loss = loss + (YO(41) * RCS(191)); \
    prod = prod + (YN(3) * (YO(40) * RCS(192))); \
    loss = loss + (YO(42) * RCS(193)); \
    prod = prod + ((YO(42) * YO(5)) * RCS(195)); \
    loss = loss + (YO(40) * RCS(194)); \
    prod = prod + ((YO(41) * YO(5)) * RCS(197)); \
    loss = loss + (YO(40) * RCS(196)); \
    prod = prod + (YN(2) * ((YO(44) * YO(38)) * RCS(225))); \
    loss = loss + (YO(43) * RCS(224)); \
    prod = prod + (((YO(5) * YO(48)) * YO(18)) * RCS(255)); \
    loss = loss + (YO(46) * RCS(254)); \
    prod = prod + 0.0; \
    loss = loss + (YO(46) * RCS(256)); \
    prod = prod + 0.0; \
    loss = loss + (YO(46) * RCS(258)); \
    prod = prod + 0.0; \
    loss = loss + (YO(46) * RCS(260)); \
    prod = prod + (((YO(5) * YO(39)) * YO(22)) * RCS(267)); \
    loss = loss + (YO(48) * RCS(266)); \
    prod = prod + (YN(2) * ((YO(5) * YO(43)) * RCS(287))); \
    loss = loss + (YO(47) * RCS(286)); \
    loss = loss + SOUR(3); \
    rhs1 = rho * Y0S(0) + dt * WM(4) * (prod + extra); \
    rhs2 = -(dt * WM(4) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(4) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(4) - fnew); \
    UC_UPDATE_TAIL(4); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 6); \
    prod = (YN(4) * (YN(0) * RCT(1, 4))); \
    extra = (1.0 * (YN(4) * (YO(46) * RCS(256)))); \
    loss = (YN(2) * RCT(1, 5)); \
    prod = prod + (YN(4) * (YOS(1) * RCT(1, 6))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(258)))); \
    loss = loss + (YN(3) * RCT(1, 7)); \
    prod = prod + (YN(4) * (YN(2) * RCT(1, 8))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    loss = loss + RCT(1, 9); \
    prod = prod + (YN(2) * (YO(6) * RCT(1, 10))); \
    loss = loss + (YN(3) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 176); \
    TM_LD(1, 1, 178); \
    TM_LD(1, 2, 240); \
    TM_LD(1, 3, 242); \
    TM_LD(1, 4, 274); \
    TM_LD(1, 5, 272); \
    TM_LD(1, 6, 284); \
    TM_LD(1, 7, 286); \
    TM_LD(1, 8, 288); \
    TM_LD(1, 9, 290); \
    TM_LD(1, 10, 312); \
    TM_LD(1, 11, 314); \
    prod = prod + (YN(4) * (YO(6) * RCT(0, 0))); \
    loss = loss + (YN(1) * RCT(0, 1)); \
    prod = prod + (YN(2) * (YO(7) * RCT(0, 2))); \
    loss = loss + (YN(4) * RCT(0, 3)); \
    prod = prod + (YN(4) * (YO(7) * RCT(0, 4))); \
    loss = loss + (YO(6) * RCT(0, 5)); \
    prod = prod + (YN(4) * (YO(10) * RCT(0, 6))); \
    loss = loss + (YO(8) * RCT(0, 7)); \
    prod = prod + (YN(4) * (YO(11) * RCT(0, 8))); \
    loss = loss + (YO(10) * RCT(0, 9)); \
    prod = prod + (YN(4) * (YO(12) * RCT(0, 10))); \
    loss = loss + (YO(13) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 352); \
    TM_LD(0, 1, 354); \
    TM_LD(0, 2, 424); \
    TM_LD(0, 3, 426); \
    TM_LD(0, 4, 492); \
    TM_LD(0, 5, 494); \
    TM_LD(0, 6, 32); \
    TM_LD(0, 7, 34); \
    TM_LD(0, 8, 36); \
    TM_LD(0, 9, 38); \
    TM_LD(0, 10, 42); \
    TM_LD(0, 11, 40); \
    prod = prod + (YN(4) * (YO(13) * RCT(1, 0))); \
    loss = loss + (YO(15) * RCT(1, 1)); \
    prod = prod + (YN(4) * (YO(14) * RCT(1, 2))); \
    loss = loss + (YO(20) * RCT(1, 3)); \
    prod = prod + (YN(2) * (YO(11) * RCT(1, 4))); \
    loss = loss + (YO(20) * RCT(1, 5)); \
    prod = prod + (YN(2) * (YO(17) * RCT(1, 6))); \
    loss = loss + (YO(15) * RCT(1, 7)); \
    prod = prod + (YN(4) * (YO(17) * RCT(1, 8))); \
    loss = loss + (YO(11) * RCT(1, 9)); \
    prod = prod + (YN(4) * (YO(19) * RCT(1, 10))); \
    loss = loss + (YO(18) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 46); \
    TM_LD(1, 1, 44); \
    TM_LD(1, 2, 50); \
    TM_LD(1, 3, 48); \
    TM_LD(1, 4, 54); \
    TM_LD(1, 5, 52); \
    TM_LD(1, 6, 58); \
    TM_LD(1, 7, 56); \
    TM_LD(1, 8, 66); \
    TM_LD(1, 9, 64); \
    TM_LD(1, 10, 68); \
    TM_LD(1, 11, 70); \
    prod = prod + (YN(4) * (YO(16) * RCT(0, 0))); \
    loss = loss + (YO(22) * RCT(0, 1)); \
    prod = prod + (YN(4) * (YO(21) * RCT(0, 2))); \
    loss = loss + (YO(27) * RCT(0, 3)); \
    prod = prod + (YN(4) * (YO(28) * RCT(0, 4))); \
    loss = loss + (YO(11) * RCT(0, 5)); \
    prod = prod + (YN(4) * (YO(29) * RCS(0))); \
    loss = loss + (YO(28) * RCS(1)); \
    prod = prod + (YN(4) * (YO(29) * RCS(2))); \
    loss = loss + (YO(17) * RCS(3)); \
    prod = prod + (YN(4) * (YO(23) * RCS(24))); \
    loss = loss + (YO(25) * RCS(25)); \
    prod = prod + (YN(4) * (YO(31) * RCS(40))); \
    loss = loss + (YO(34) * RCS(41)); \
    prod = prod + (YN(4) * (YO(31) * RCS(42))); \
    loss = loss + (YO(23) * RCS(43)); \
    prod = prod + (YO(30) * RCS(64)); \
    loss = loss + (YO(16) * RCS(65)); \
    prod = prod + (YN(4) * (YO(30) * RCS(66))); \
    loss = loss + (YO(33) * RCS(67)); \
    prod = prod + (YN(4) * (YO(30) * RCS(68))); \
    loss = loss + (YO(32) * RCS(69)); \
    prod = prod + (YN(4) * (YO(30) * RCS(70))); \
    loss = loss + (YO(35) * RCS(71)); \
    prod = prod + (YN(2) * (YO(35) * RCS(110))); \
    loss = loss + (YO(16) * RCS(111)); \
    prod = prod + (YN(4) * (YO(35) * RCS(112))); \
    loss = loss + (YO(31) * RCS(113)); \
    prod = prod + (YN(2) * (YO(32) * RCS(118))); \
    loss = loss + (YO(16) * RCS(119)); \
    prod = prod + (YN(4) * (YO(32) * RCS(124))); \
    loss = loss + (YO(31) * RCS(125)); \
    prod = prod + (YN(4) * (YO(36) * RCS(138))); \
    loss = loss + (YO(37) * RCS(139)); \
    prod = prod + (YN(4) * (YO(38) * RCS(152))); \
    loss = loss + (YO(36) * RCS(153)); \
    prod = prod + (YN(4) * (YO(39) * RCS(162))); \
    loss = loss + (YO(38) * RCS(163)); \
    prod = prod + (YN(4) * (YO(40) * RCS(194))); \
    loss = loss + (YO(42) * RCS(195)); \
    prod = prod + (YN(4) * (YO(40) * RCS(196))); \
    loss = loss + (YO(41) * RCS(197)); \
    prod = prod + (YN(4) * (YO(46) * RCS(254))); \
    loss = loss + ((YO(48) * YO(18)) * RCS(255)); \
    prod = prod + (YN(4) * (YO(48) * RCS(266))); \
    loss = loss + ((YO(39) * YO(22)) * RCS(267)); \
    prod = prod + (YN(4) * (YO(47) * RCS(286))); \
    loss = loss + ((YO(43) * YN(2)) * RCS(287)); \
    rhs1 = rho * Y0S(1) + dt * WM(5) * (prod + extra); \
    rhs2 = -(dt * WM(5) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(5) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(5) - fnew); \
    UC_UPDATE_TAIL(5); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 7); \
    prod = (YN(4) * (YN(3) * RCT(0, 6))); \
    extra = 0.0; \
    loss = RCT(0, 7); \
    prod = prod + (YN(2) * (YN(1) * RCT(0, 8))); \
    loss = loss + RCT(0, 9); \
    prod = prod + (YN(4) * (YOS(1) * RCT(0, 10))); \
    loss = loss + (YN(2) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 76); \
    TM_LD(0, 1, 78); \
    TM_LD(0, 2, 80); \
    TM_LD(0, 3, 82); \
    TM_LD(0, 4, 90); \
    TM_LD(0, 5, 88); \
    TM_LD(0, 6, 116); \
    TM_LD(0, 7, 118); \
    TM_LD(0, 8, 140); \
    TM_LD(0, 9, 142); \
    TM_LD(0, 10, 146); \
    TM_LD(0, 11, 144); \
    prod = prod + (YN(1) * (YN(0) * RCT(1, 0))); \
    loss = loss + (YN(2) * RCT(1, 1)); \
    prod = prod + (YN(5) * (YN(3) * RCT(1, 2))); \
    loss = loss + (YN(2) * RCT(1, 3)); \
    prod = prod + (YN(4) * (YN(1) * RCT(1, 4))); \
    loss = loss + (YN(3) * RCT(1, 5)); \
    prod = prod + (YN(5) * (YN(1) * RCT(1, 6))); \
    loss = loss + (YN(4) * RCT(1, 7)); \
    prod = prod + (YN(1) * (YO(7) * RCT(1, 8))); \
    loss = loss + (YO(6) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(7) * RCT(1, 8))); \
    loss = loss + (YO(6) * RCT(1, 9)); \
    prod = prod + (YN(2) * (YO(7) * RCT(1, 10))); \
    loss = loss + (YN(0) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 160); \
    TM_LD(1, 1, 162); \
    TM_LD(1, 2, 166); \
    TM_LD(1, 3, 164); \
    TM_LD(1, 4, 190); \
    TM_LD(1, 5, 188); \
    TM_LD(1, 6, 296); \
    TM_LD(1, 7, 298); \
    TM_LD(1, 8, 326); \
    TM_LD(1, 9, 324); \
    TM_LD(1, 10, 340); \
    TM_LD(1, 11, 342); \
    prod = prod + (YN(4) * (YO(7) * RCT(0, 0))); \
    loss = loss + (YN(5) * RCT(0, 1)); \
    prod = prod + (YN(3) * (YO(7) * RCT(0, 2))); \
    loss = loss + (YN(4) * RCT(0, 3)); \
    prod = prod + (YN(4) * (YO(9) * RCT(0, 4))); \
    loss = loss + (YO(8) * RCT(0, 5)); \
    prod = prod + (YN(1) * (YO(10) * RCT(0, 6))); \
    loss = loss + (YO(8) * RCT(0, 7)); \
    prod = prod + (YN(1) * (YO(11) * RCT(0, 8))); \
    loss = loss + (YO(10) * RCT(0, 9)); \
    prod = prod + ((YO(10) * YO(7)) * RCT(0, 10)); \
    loss = loss + (YO(11) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 368); \
    TM_LD(0, 1, 370); \
    TM_LD(0, 2, 374); \
    TM_LD(0, 3, 372); \
    TM_LD(0, 4, 378); \
    TM_LD(0, 5, 376); \
    TM_LD(0, 6, 404); \
    TM_LD(0, 7, 406); \
    TM_LD(0, 8, 496); \
    TM_LD(0, 9, 498); \
    TM_LD(0, 10, 60); \
    TM_LD(0, 11, 62); \
    prod = prod + (YN(1) * (YO(12) * RCT(1, 0))); \
    loss = loss + (YO(13) * RCT(1, 1)); \
    prod = prod + ((YO(13) * YO(7)) * RCT(1, 2)); \
    loss = loss + (YO(12) * RCT(1, 3)); \
    prod = prod + (YN(4) * (YO(17) * RCT(1, 4))); \
    loss = loss + (YO(13) * RCT(1, 5)); \
    prod = prod + (YN(1) * (YO(17) * RCT(1, 6))); \
    loss = loss + (YO(11) * RCT(1, 7)); \
    prod = prod + ((YO(18) * YO(7)) * RCT(1, 8)); \
    loss = loss + (YO(19) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(18) * RCT(1, 10))); \
    loss = loss + (YO(16) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 64); \
    TM_LD(1, 1, 66); \
    TM_LD(1, 2, 70); \
    TM_LD(1, 3, 68); \
    TM_LD(1, 4, 74); \
    TM_LD(1, 5, 72); \
    TM_LD(1, 6, 78); \
    TM_LD(1, 7, 76); \
    TM_LD(1, 8, 82); \
    TM_LD(1, 9, 80); \
    TM_LD(1, 10, 144); \
    TM_LD(1, 11, 146); \
    prod = prod + (YN(1) * (YO(16) * RCT(0, 0))); \
    loss = loss + (YO(22) * RCT(0, 1)); \
    prod = prod + (YN(4) * (YO(24) * RCT(0, 2))); \
    loss = loss + (YO(16) * RCT(0, 3)); \
    prod = prod + (((YO(13) * YO(8)) * YO(7)) * RCT(0, 4)); \
    loss = loss + (YO(24) * RCT(0, 5)); \
    prod = prod + (YN(1) * (YO(22) * RCT(0, 6))); \
    loss = loss + (YO(21) * RCT(0, 7)); \
    prod = prod + (YN(1) * (YO(28) * RCT(0, 8))); \
    loss = loss + (YO(11) * RCT(0, 9)); \
    prod = prod + ((YO(28) * YO(7)) * RCS(11)); \
    loss = loss + (YO(29) * RCS(10)); \
    prod = prod + (YN(1) * (YO(29) * RCS(12))); \
    loss = loss + (YO(28) * RCS(13)); \
    prod = prod + (YN(4) * ((YO(11) * YO(10)) * RCS(31))); \
    loss = loss + (YO(23) * RCS(30)); \
    prod = prod + (YN(1) * (YO(31) * RCS(33))); \
    loss = loss + (YO(23) * RCS(32)); \
    prod = prod + ((YO(34) * YO(7)) * RCS(57)); \
    loss = loss + (YO(31) * RCS(56)); \
    prod = prod + ((YO(23) * YO(7)) * RCS(59)); \
    loss = loss + (YO(31) * RCS(58)); \
    prod = prod + (YN(1) * (YO(31) * RCS(60))); \
    loss = loss + (YO(34) * RCS(61)); \
    prod = prod + ((YO(32) * YO(7)) * RCS(91)); \
    loss = loss + (YO(30) * RCS(90)); \
    prod = prod + ((YO(33) * YO(7)) * RCS(93)); \
    loss = loss + (YO(30) * RCS(92)); \
    prod = prod + ((YO(35) * YO(7)) * RCS(95)); \
    loss = loss + (YO(30) * RCS(94)); \
    prod = prod + (YN(4) * (YO(35) * RCS(99))); \
    loss = loss + (YO(18) * RCS(98)); \
    prod = prod + (YN(1) * (YO(35) * RCS(104))); \
    loss = loss + (YO(31) * RCS(105)); \
    prod = prod + (YN(1) * (YO(32) * RCS(114))); \
    loss = loss + (YO(31) * RCS(115)); \
    prod = prod + (YN(4) * ((YO(31) * YOS(1)) * RCS(123))); \
    loss = loss + (YO(32) * RCS(122)); \
    prod = prod + (YN(1) * (YO(36) * RCS(137))); \
    loss = loss + (YO(37) * RCS(136)); \
    prod = prod + (YN(1) * (YO(38) * RCS(146))); \
    loss = loss + (YO(36) * RCS(147)); \
    prod = prod + (YN(4) * ((YO(8) * YO(22)) * RCS(157))); \
    loss = loss + (YO(37) * RCS(156)); \
    prod = prod + (YN(1) * (YO(39) * RCS(171))); \
    loss = loss + (YO(38) * RCS(170)); \
    prod = prod + (YN(4) * ((YO(22) * YO(11)) * RCS(173))); \
    loss = loss + (YO(38) * RCS(172)); \
    prod = prod + (YN(1) * (YO(40) * RCS(182))); \
    loss = loss + (YO(41) * RCS(183)); \
    prod = prod + (YN(1) * (YO(40) * RCS(184))); \
    loss = loss + (YO(42) * RCS(185)); \
    prod = prod + ((YO(41) * YO(7)) * RCS(199)); \
    loss = loss + (YO(40) * RCS(198)); \
    prod = prod + ((YO(42) * YO(7)) * RCS(201)); \
    loss = loss + (YO(40) * RCS(200)); \
    prod = prod + (YN(1) * (YO(41) * RCS(206))); \
    loss = loss + (YO(39) * RCS(207)); \
    prod = prod + (YN(1) * (YO(42) * RCS(212))); \
    loss = loss + (YO(39) * RCS(213)); \
    prod = prod + (YN(1) * (YO(45) * RCS(236))); \
    loss = loss + ((YO(21) * YO(38)) * RCS(237)); \
    prod = prod + (YN(1) * (YO(45) * RCS(238))); \
    loss = loss + ((YO(22) * YO(36)) * RCS(239)); \
    prod = prod + (((YO(21) * YO(38)) * YO(7)) * RCS(241)); \
    loss = loss + (YO(45) * RCS(240)); \
    prod = prod + (((YO(22) * YO(36)) * YO(7)) * RCS(243)); \
    loss = loss + (YO(45) * RCS(242)); \
    rhs1 = rho * Y0S(0) + dt * WM(6) * (prod + extra); \
    rhs2 = -(dt * WM(6) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(6) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(6) - fnew); \
    UC_UPDATE_TAIL(6); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 8); \
    prod = (YN(4) * (YOS(1) * RCT(0, 10))); \
    extra = 0.0; \
    loss = RCT(0, 11); \
    TM_WAIT(1); \
    TM_LD(0, 0, 164); \
    TM_LD(0, 1, 166); \
    TM_LD(0, 2, 324); \
    TM_LD(0, 3, 326); \
    TM_LD(0, 4, 376); \
    TM_LD(0, 5, 378); \
    TM_LD(0, 6, 86); \
    TM_LD(0, 7, 84); \
    TM_LD(0, 8, 90); \
    TM_LD(0, 9, 88); \
    TM_LD(0, 10, 94); \
    TM_LD(0, 11, 92); \
    prod = prod + (YN(6) * (YOS(2) * RCT(1, 0))); \
    loss = loss + (YN(1) * RCT(1, 1)); \
    prod = prod + (YN(6) * (YN(0) * RCT(1, 2))); \
    loss = loss + (YN(2) * RCT(1, 3)); \
    prod = prod + (YN(5) * (YN(4) * RCT(1, 4))); \
    loss = loss + (YN(2) * RCT(1, 5)); \
    prod = prod + (YN(6) * (YN(5) * RCT(1, 6))); \
    loss = loss + (YN(4) * RCT(1, 7)); \
    prod = prod + (YN(6) * (YN(4) * RCT(1, 8))); \
    loss = loss + (YN(3) * RCT(1, 9)); \
    prod = prod + (YN(6) * (YO(11) * RCT(1, 10))); \
    loss = loss + (YO(10) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 96); \
    TM_LD(1, 1, 98); \
    TM_LD(1, 2, 100); \
    TM_LD(1, 3, 102); \
    TM_LD(1, 4, 104); \
    TM_LD(1, 5, 106); \
    TM_LD(1, 6, 112); \
    TM_LD(1, 7, 114); \
    TM_LD(1, 8, 116); \
    TM_LD(1, 9, 118); \
    TM_LD(1, 10, 120); \
    TM_LD(1, 11, 122); \
    prod = prod + (YN(6) * (YO(12) * RCT(0, 0))); \
    loss = loss + (YO(13) * RCT(0, 1)); \
    prod = prod + (YN(6) * (YO(19) * RCT(0, 2))); \
    loss = loss + (YO(18) * RCT(0, 3)); \
    prod = prod + (YN(6) * (YO(24) * RCT(0, 4))); \
    loss = loss + ((YO(13) * YO(8)) * RCT(0, 5)); \
    prod = prod + (YN(6) * (YO(29) * RCS(10))); \
    loss = loss + (YO(28) * RCS(11)); \
    prod = prod + (YN(6) * (YO(31) * RCS(56))); \
    loss = loss + (YO(34) * RCS(57)); \
    prod = prod + (YN(6) * (YO(31) * RCS(58))); \
    loss = loss + (YO(23) * RCS(59)); \
    prod = prod + (YN(6) * (YO(30) * RCS(90))); \
    loss = loss + (YO(32) * RCS(91)); \
    prod = prod + (YN(6) * (YO(30) * RCS(92))); \
    loss = loss + (YO(33) * RCS(93)); \
    prod = prod + (YN(6) * (YO(30) * RCS(94))); \
    loss = loss + (YO(35) * RCS(95)); \
    prod = prod + (YN(6) * (YO(40) * RCS(198))); \
    loss = loss + (YO(41) * RCS(199)); \
    prod = prod + (YN(6) * (YO(40) * RCS(200))); \
    loss = loss + (YO(42) * RCS(201)); \
    prod = prod + (YN(6) * (YO(45) * RCS(240))); \
    loss = loss + ((YO(21) * YO(38)) * RCS(241)); \
    prod = prod + (YN(6) * (YO(45) * RCS(242))); \
    loss = loss + ((YO(22) * YO(36)) * RCS(243)); \
    rhs1 = rho * Y0S(1) + dt * WM(7) * (prod + extra); \
    rhs2 = -(dt * WM(7) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(7) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(7) - fnew); \
    UC_UPDATE_TAIL(7); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 9); \
    prod = (YN(2) * (YO(9) * RCT(0, 6))); \
    extra = 0.0; \
    loss = (YN(4) * RCT(0, 7)); \
    prod = prod + (YN(4) * (YO(9) * RCT(0, 8))); \
    loss = loss + (YN(6) * RCT(0, 9)); \
    prod = prod + (YN(3) * (YO(9) * RCT(0, 10))); \
    loss = loss + (YN(1) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 220); \
    TM_LD(0, 1, 222); \
    TM_LD(0, 2, 224); \
    TM_LD(0, 3, 226); \
    TM_LD(0, 4, 244); \
    TM_LD(0, 5, 246); \
    TM_LD(0, 6, 248); \
    TM_LD(0, 7, 250); \
    TM_LD(0, 8, 256); \
    TM_LD(0, 9, 258); \
    TM_LD(0, 10, 264); \
    TM_LD(0, 11, 266); \
    prod = prod + (YO(10) * RCT(1, 0)); \
    loss = loss + (YN(2) * RCT(1, 1)); \
    prod = prod + (YN(2) * (YO(10) * RCT(1, 2))); \
    loss = loss + (YN(0) * RCT(1, 3)); \
    prod = prod + (YN(3) * (YO(10) * RCT(1, 4))); \
    loss = loss + (YN(4) * RCT(1, 5)); \
    prod = prod + (YN(4) * (YO(10) * RCT(1, 6))); \
    loss = loss + (YN(5) * RCT(1, 7)); \
    prod = prod + (YN(1) * (YO(10) * RCT(1, 8))); \
    loss = loss + (YN(6) * RCT(1, 9)); \
    prod = prod + ((YO(10) * YO(13)) * RCT(1, 10)); \
    loss = loss + (YO(12) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 276); \
    TM_LD(1, 1, 278); \
    TM_LD(1, 2, 376); \
    TM_LD(1, 3, 378); \
    TM_LD(1, 4, 412); \
    TM_LD(1, 5, 414); \
    TM_LD(1, 6, 416); \
    TM_LD(1, 7, 418); \
    TM_LD(1, 8, 428); \
    TM_LD(1, 9, 430); \
    TM_LD(1, 10, 440); \
    TM_LD(1, 11, 442); \
    prod = prod + (YN(1) * (YO(15) * RCT(0, 0))); \
    loss = loss + ((YN(4) * YN(2)) * RCT(0, 1)); \
    prod = prod + ((YO(15) * YO(9)) * RCT(0, 2)); \
    loss = loss + (YO(11) * RCT(0, 3)); \
    prod = prod + (YN(3) * (YO(14) * RCT(0, 4))); \
    loss = loss + ((YN(2) * YN(2)) * RCT(0, 5)); \
    prod = prod + (YN(3) * (YO(14) * RCT(0, 6))); \
    loss = loss + (YN(0) * RCT(0, 7)); \
    prod = prod + (YN(1) * (YO(14) * RCT(0, 8))); \
    loss = loss + ((YN(4) * YN(2)) * RCT(0, 9)); \
    prod = prod + (YN(3) * (YO(20) * RCT(0, 10))); \
    loss = loss + (YN(2) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 444); \
    TM_LD(0, 1, 446); \
    TM_LD(0, 2, 448); \
    TM_LD(0, 3, 450); \
    TM_LD(0, 4, 452); \
    TM_LD(0, 5, 454); \
    TM_LD(0, 6, 456); \
    TM_LD(0, 7, 458); \
    TM_LD(0, 8, 460); \
    TM_LD(0, 9, 462); \
    TM_LD(0, 10, 468); \
    TM_LD(0, 11, 470); \
    prod = prod + ((YO(20) * YO(9)) * RCT(1, 0)); \
    loss = loss + (YO(10) * RCT(1, 1)); \
    prod = prod + (YN(6) * (YO(24) * RCT(1, 2))); \
    loss = loss + ((YO(13) * YN(7)) * RCT(1, 3)); \
    prod = prod + (YN(3) * (YO(21) * RCT(1, 4))); \
    loss = loss + (YO(14) * RCT(1, 5)); \
    prod = prod + (YN(1) * (YO(21) * RCT(1, 6))); \
    loss = loss + (YO(11) * RCT(1, 7)); \
    prod = prod + (YN(2) * (YO(25) * RCT(1, 8))); \
    loss = loss + (YO(13) * RCT(1, 9)); \
    prod = prod + ((YO(25) * YO(13)) * RCT(1, 10)); \
    loss = loss + (YO(18) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 480); \
    TM_LD(1, 1, 482); \
    TM_LD(1, 2, 508); \
    TM_LD(1, 3, 510); \
    TM_LD(1, 4, 84); \
    TM_LD(1, 5, 86); \
    TM_LD(1, 6, 88); \
    TM_LD(1, 7, 90); \
    TM_LD(1, 8, 92); \
    TM_LD(1, 9, 94); \
    TM_LD(1, 10, 108); \
    TM_LD(1, 11, 110); \
    prod = prod + (YN(2) * (YO(26) * RCT(0, 0))); \
    loss = loss + (YO(15) * RCT(0, 1)); \
    prod = prod + (YN(4) * (YO(26) * RCT(0, 2))); \
    loss = loss + ((YO(10) * YN(2)) * RCT(0, 3)); \
    prod = prod + (YN(3) * (YO(26) * RCT(0, 4))); \
    loss = loss + ((YO(8) * YN(2)) * RCT(0, 5)); \
    prod = prod + (YN(3) * (YO(26) * RCT(0, 4))); \
    loss = loss + ((YO(8) * YN(2)) * RCT(0, 5)); \
    prod = prod + (YN(1) * (YO(26) * RCT(0, 6))); \
    loss = loss + ((YO(8) * YN(4)) * RCT(0, 7)); \
    prod = prod + (YN(1) * (YO(26) * RCT(0, 6))); \
    loss = loss + ((YO(8) * YN(4)) * RCT(0, 7)); \
    prod = prod + (YN(1) * (YO(26) * RCT(0, 8))); \
    loss = loss + ((YO(9) * YN(2)) * RCT(0, 9)); \
    prod = prod + (YN(3) * (YO(27) * RCT(0, 10))); \
    loss = loss + (YO(20) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 226); \
    TM_LD(0, 1, 224); \
    TM_LD(0, 2, 252); \
    TM_LD(0, 3, 254); \
    TM_LD(0, 4, 278); \
    TM_LD(0, 5, 276); \
    TM_LD(0, 6, 432); \
    TM_LD(0, 7, 434); \
    TM_LD(0, 8, 460); \
    TM_LD(0, 9, 462); \
    TM_LD(0, 10, 476); \
    TM_LD(0, 11, 478); \
    prod = prod + (YN(1) * (YO(27) * RCT(1, 0))); \
    loss = loss + (YO(10) * RCT(1, 1)); \
    prod = prod + (YN(4) * (YO(25) * RCT(1, 2))); \
    loss = loss + (YO(28) * RCT(1, 3)); \
    prod = prod + (YN(1) * (YO(23) * RCS(26))); \
    loss = loss + ((YO(11) * YN(4)) * RCS(27)); \
    prod = prod + ((YO(23) * YO(13)) * RCS(28)); \
    loss = loss + ((YO(18) * YN(2)) * RCS(29)); \
    prod = prod + (YO(23) * RCS(34)); \
    loss = loss + (YO(13) * RCS(35)); \
    prod = prod + (YO(34) * RCS(38)); \
    loss = loss + (YO(13) * RCS(39)); \
    prod = prod + ((YO(18) * YO(9)) * RCS(107)); \
    loss = loss + (YO(35) * RCS(106)); \
    prod = prod + (YN(3) * (YO(36) * RCS(128))); \
    loss = loss + (YO(16) * RCS(129)); \
    prod = prod + ((YO(37) * YO(10)) * RCS(154)); \
    loss = loss + (YO(36) * RCS(155)); \
    prod = prod + (YN(6) * (YO(37) * RCS(156))); \
    loss = loss + ((YN(4) * YO(22)) * RCS(157)); \
    prod = prod + (YN(1) * (YO(36) * RCS(158))); \
    loss = loss + ((YO(13) * YO(10)) * RCS(159)); \
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
    prod = (YN(8) * (YN(4) * RCT(1, 4))); \
    extra = 0.0; \
    loss = (YN(2) * RCT(1, 5)); \
    prod = prod + (YN(8) * (YN(6) * RCT(1, 6))); \
    loss = loss + (YN(4) * RCT(1, 7)); \
    prod = prod + (YN(8) * (YN(1) * RCT(1, 8))); \
    loss = loss + (YN(3) * RCT(1, 9)); \
    prod = prod + (YN(3) * (YO(10) * RCT(1, 10))); \
    loss = loss + (YN(2) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 98); \
    TM_LD(1, 1, 96); \
    TM_LD(1, 2, 102); \
    TM_LD(1, 3, 100); \
    TM_LD(1, 4, 106); \
    TM_LD(1, 5, 104); \
    TM_LD(1, 6, 110); \
    TM_LD(1, 7, 108); \
    TM_LD(1, 8, 114); \
    TM_LD(1, 9, 112); \
    TM_LD(1, 10, 118); \
    TM_LD(1, 11, 116); \
    prod = prod + (YN(8) * (YO(11) * RCT(0, 0))); \
    loss = loss + (YO(15) * RCT(0, 1)); \
    prod = prod + (YN(1) * (YO(14) * RCT(0, 2))); \
    loss = loss + (YN(0) * RCT(0, 3)); \
    prod = prod + (YN(8) * (YO(10) * RCT(0, 4))); \
    loss = loss + (YO(20) * RCT(0, 5)); \
    prod = prod + (YN(3) * (YO(25) * RCT(0, 6))); \
    loss = loss + (YO(14) * RCT(0, 7)); \
    prod = prod + (YN(1) * (YO(26) * RCT(0, 8))); \
    loss = loss + ((YN(8) * YN(2)) * RCT(0, 9)); \
    prod = prod + (YN(1) * (YO(27) * RCT(0, 10))); \
    loss = loss + (YO(20) * RCT(0, 11)); \
    prod = prod + (YN(8) * (YO(35) * RCS(106))); \
    loss = loss + (YO(18) * RCS(107)); \
    rhs1 = rho * Y0S(1) + dt * WM(9) * (prod + extra); \
    rhs2 = -(dt * WM(9) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(9) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(9) - fnew); \
    UC_UPDATE_TAIL(9); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 11); \
    TM_WAIT(1); \
    TM_LD(0, 0, 122); \
    TM_LD(0, 1, 120); \
    TM_LD(0, 2, 126); \
    TM_LD(0, 3, 124); \
    TM_LD(0, 4, 128); \
    TM_LD(0, 5, 130); \
    TM_LD(0, 6, 132); \
    TM_LD(0, 7, 134); \
    TM_LD(0, 8, 136); \
    TM_LD(0, 9, 138); \
    TM_LD(0, 10, 140); \
    TM_LD(0, 11, 142); \
    prod = (YN(8) * (YN(2) * RCT(1, 0))); \
    extra = 0.0; \
    loss = RCT(1, 1); \
    prod = prod + (YN(8) * (YN(0) * RCT(1, 2))); \
    loss = loss + (YN(2) * RCT(1, 3)); \
    prod = prod + (YN(8) * (YN(4) * RCT(1, 4))); \
    loss = loss + (YN(3) * RCT(1, 5)); \
    prod = prod + (YN(9) * (YN(2) * RCT(1, 6))); \
    loss = loss + (YN(3) * RCT(1, 7)); \
    prod = prod + (YN(8) * (YN(5) * RCT(1, 8))); \
    loss = loss + (YN(4) * RCT(1, 9)); \
    prod = prod + (YN(8) * (YN(6) * RCT(1, 10))); \
    loss = loss + (YN(1) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 144); \
    TM_LD(1, 1, 146); \
    TM_LD(1, 2, 268); \
    TM_LD(1, 3, 270); \
    TM_LD(1, 4, 276); \
    TM_LD(1, 5, 278); \
    TM_LD(1, 6, 356); \
    TM_LD(1, 7, 358); \
    TM_LD(1, 8, 396); \
    TM_LD(1, 9, 398); \
    TM_LD(1, 10, 448); \
    TM_LD(1, 11, 450); \
    prod = prod + (YN(8) * (YO(12) * RCT(0, 0))); \
    loss = loss + (YO(13) * RCT(0, 1)); \
    prod = prod + (YO(11) * RCT(0, 2)); \
    loss = loss + (YN(2) * RCT(0, 3)); \
    prod = prod + (YN(2) * (YO(11) * RCT(0, 4))); \
    loss = loss + (YN(0) * RCT(0, 5)); \
    prod = prod + (YN(3) * (YO(11) * RCT(0, 6))); \
    loss = loss + (YN(4) * RCT(0, 7)); \
    prod = prod + (YN(4) * (YO(11) * RCT(0, 8))); \
    loss = loss + (YN(5) * RCT(0, 9)); \
    prod = prod + (YN(1) * (YO(11) * RCT(0, 10))); \
    loss = loss + (YN(6) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 480); \
    TM_LD(0, 1, 482); \
    TM_LD(0, 2, 124); \
    TM_LD(0, 3, 126); \
    TM_LD(0, 4, 130); \
    TM_LD(0, 5, 128); \
    TM_LD(0, 6, 134); \
    TM_LD(0, 7, 132); \
    TM_LD(0, 8, 138); \
    TM_LD(0, 9, 136); \
    TM_LD(0, 10, 142); \
    TM_LD(0, 11, 140); \
    prod = prod + (YN(6) * (YO(11) * RCT(1, 0))); \
    loss = loss + (YN(7) * RCT(1, 1)); \
    prod = prod + (YN(1) * (YO(20) * RCT(1, 2))); \
    loss = loss + (YN(3) * RCT(1, 3)); \
    prod = prod + (YN(9) * (YO(20) * RCT(1, 4))); \
    loss = loss + (YN(8) * RCT(1, 5)); \
    prod = prod + (YN(3) * (YO(16) * RCT(1, 6))); \
    loss = loss + (YO(13) * RCT(1, 7)); \
    prod = prod + (YN(1) * (YO(22) * RCT(1, 8))); \
    loss = loss + (YO(11) * RCT(1, 9)); \
    prod = prod + (YN(4) * (YO(26) * RCT(1, 10))); \
    loss = loss + ((YN(8) * YN(2)) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 146); \
    TM_LD(1, 1, 144); \
    TM_LD(1, 2, 180); \
    TM_LD(1, 3, 182); \
    TM_LD(1, 4, 192); \
    TM_LD(1, 5, 194); \
    TM_LD(1, 6, 216); \
    TM_LD(1, 7, 218); \
    TM_LD(1, 8, 224); \
    TM_LD(1, 9, 226); \
    TM_LD(1, 10, 236); \
    TM_LD(1, 11, 238); \
    prod = prod + (YN(1) * (YO(27) * RCT(0, 0))); \
    loss = loss + (YN(8) * RCT(0, 1)); \
    prod = prod + (YN(2) * (YO(23) * RCS(18))); \
    loss = loss + (YO(13) * RCS(19)); \
    prod = prod + (YN(3) * (YO(23) * RCS(22))); \
    loss = loss + (YO(11) * RCS(23)); \
    prod = prod + (YN(6) * (YO(23) * RCS(30))); \
    loss = loss + ((YO(11) * YN(4)) * RCS(31)); \
    prod = prod + (YO(31) * RCS(36)); \
    loss = loss + (YO(13) * RCS(37)); \
    prod = prod + (YN(1) * (YO(37) * RCS(140))); \
    loss = loss + (YO(25) * RCS(141)); \
    prod = prod + (YN(8) * (YO(36) * RCS(155))); \
    loss = loss + (YO(37) * RCS(154)); \
    prod = prod + (YN(1) * (YO(36) * RCS(158))); \
    loss = loss + ((YO(13) * YN(8)) * RCS(159)); \
    prod = prod + (YN(3) * (YO(39) * RCS(160))); \
    loss = loss + (YO(18) * RCS(161)); \
    rhs1 = rho * Y0S(0) + dt * WM(10) * (prod + extra); \
    rhs2 = -(dt * WM(10) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(10) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(10) - fnew); \
    UC_UPDATE_TAIL(10); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 12); \
    prod = (YN(10) * (YN(2) * RCT(0, 2))); \
    extra = 0.0; \
    loss = RCT(0, 3); \
    prod = prod + (YN(10) * (YN(0) * RCT(0, 4))); \
    loss = loss + (YN(2) * RCT(0, 5)); \
    prod = prod + (YN(10) * (YN(4) * RCT(0, 6))); \
    loss = loss + (YN(3) * RCT(0, 7)); \
    prod = prod + (YN(10) * (YN(5) * RCT(0, 8))); \
    loss = loss + (YN(4) * RCT(0, 9)); \
    prod = prod + (YN(10) * (YN(6) * RCT(0, 10))); \
    loss = loss + (YN(1) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 272); \
    TM_LD(0, 1, 274); \
    TM_LD(0, 2, 280); \
    TM_LD(0, 3, 282); \
    TM_LD(0, 4, 288); \
    TM_LD(0, 5, 290); \
    TM_LD(0, 6, 292); \
    TM_LD(0, 7, 294); \
    TM_LD(0, 8, 296); \
    TM_LD(0, 9, 298); \
    TM_LD(0, 10, 300); \
    TM_LD(0, 11, 302); \
    prod = prod + (YN(10) * (YN(7) * RCT(1, 0))); \
    loss = loss + (YN(6) * RCT(1, 1)); \
    prod = prod + (YN(3) * (YO(13) * RCT(1, 2))); \
    loss = loss + (YN(2) * RCT(1, 3)); \
    prod = prod + (YN(1) * (YO(13) * RCT(1, 4))); \
    loss = loss + (YN(4) * RCT(1, 5)); \
    prod = prod + (YN(4) * (YO(15) * RCT(1, 6))); \
    loss = loss + (YN(2) * RCT(1, 7)); \
    prod = prod + (YN(9) * (YO(15) * RCT(1, 8))); \
    loss = loss + (YN(8) * RCT(1, 9)); \
    prod = prod + (YN(4) * (YO(14) * RCT(1, 10))); \
    loss = loss + (YN(2) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 336); \
    TM_LD(1, 1, 338); \
    TM_LD(1, 2, 396); \
    TM_LD(1, 3, 398); \
    TM_LD(1, 4, 416); \
    TM_LD(1, 5, 418); \
    TM_LD(1, 6, 484); \
    TM_LD(1, 7, 486); \
    TM_LD(1, 8, 492); \
    TM_LD(1, 9, 494); \
    TM_LD(1, 10, 496); \
    TM_LD(1, 11, 498); \
    prod = prod + (YN(5) * (YO(20) * RCT(0, 0))); \
    loss = loss + (YN(2) * RCT(0, 1)); \
    prod = prod + (YN(2) * (YO(17) * RCT(0, 2))); \
    loss = loss + (YN(0) * RCT(0, 3)); \
    prod = prod + (YN(4) * (YO(17) * RCT(0, 4))); \
    loss = loss + (YN(5) * RCT(0, 5)); \
    prod = prod + (YN(3) * (YO(17) * RCT(0, 6))); \
    loss = loss + (YN(4) * RCT(0, 7)); \
    prod = prod + (YN(1) * (YO(17) * RCT(0, 8))); \
    loss = loss + (YN(6) * RCT(0, 9)); \
    prod = prod + (YO(17) * RCT(0, 10)); \
    loss = loss + (YN(2) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 500); \
    TM_LD(0, 1, 502); \
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
    prod = prod + (YN(3) * (YO(18) * RCT(1, 0))); \
    loss = loss + (YO(13) * RCT(1, 1)); \
    prod = prod + (YN(1) * (YO(22) * RCT(1, 2))); \
    loss = loss + (YN(10) * RCT(1, 3)); \
    prod = prod + (YN(1) * (YO(21) * RCT(1, 4))); \
    loss = loss + (YN(8) * RCT(1, 5)); \
    prod = prod + (YN(2) * (YO(28) * RCT(1, 6))); \
    loss = loss + (YN(0) * RCT(1, 7)); \
    prod = prod + (YN(4) * (YO(28) * RCT(1, 8))); \
    loss = loss + (YN(5) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(28) * RCT(1, 10))); \
    loss = loss + (YN(6) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 166); \
    TM_LD(1, 1, 164); \
    TM_LD(1, 2, 208); \
    TM_LD(1, 3, 210); \
    TM_LD(1, 4, 316); \
    TM_LD(1, 5, 318); \
    TM_LD(1, 6, 122); \
    TM_LD(1, 7, 120); \
    TM_LD(1, 8, 148); \
    TM_LD(1, 9, 150); \
    TM_LD(1, 10, 152); \
    TM_LD(1, 11, 154); \
    prod = prod + (YO(28) * RCT(0, 0)); \
    loss = loss + (YN(2) * RCT(0, 1)); \
    prod = prod + (YN(3) * (YO(23) * RCS(22))); \
    loss = loss + (YN(10) * RCS(23)); \
    prod = prod + (YN(1) * (YO(23) * RCS(26))); \
    loss = loss + ((YN(8) * YN(4)) * RCS(27)); \
    prod = prod + (YN(6) * (YO(23) * RCS(30))); \
    loss = loss + ((YN(10) * YN(4)) * RCS(31)); \
    prod = prod + (YO(35) * RCS(102)); \
    loss = loss + (YO(13) * RCS(103)); \
    prod = prod + (YN(6) * (YO(38) * RCS(172))); \
    loss = loss + ((YN(4) * YO(22)) * RCS(173)); \
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
    prod = prod + ((YO(31) * YO(13)) * RCS(52)); \
    loss = loss + (YO(34) * RCS(53)); \
    prod = prod + ((YO(31) * YO(13)) * RCS(54)); \
    loss = loss + (YO(23) * RCS(55)); \
    prod = prod + ((YO(30) * YO(13)) * RCS(84)); \
    loss = loss + (YO(33) * RCS(85)); \
    prod = prod + ((YO(30) * YO(13)) * RCS(86)); \
    loss = loss + (YO(32) * RCS(87)); \
    prod = prod + ((YO(30) * YO(13)) * RCS(88)); \
    loss = loss + (YO(35) * RCS(89)); \
    prod = prod + ((YO(38) * YO(13)) * RCS(148)); \
    loss = loss + (YO(36) * RCS(149)); \
    prod = prod + ((YO(43) * YO(13)) * RCS(226)); \
    loss = loss + ((YO(21) * YO(22)) * RCS(227)); \
    rhs1 = rho * Y0S(0) + dt * WM(12) * (prod + extra); \
    rhs2 = -(dt * WM(12) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(12) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(12) - fnew); \
    UC_UPDATE_TAIL(12); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 14); \
    prod = (YN(12) * (YN(8) * RCT(1, 6))); \
    extra = (1.0 * (YO(46) * RCS(244))); \
    loss = (YN(10) * RCT(1, 7)); \
    prod = prod + (YN(12) * (YN(2) * RCT(1, 8))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(248)))); \
    loss = loss + (YN(0) * RCT(1, 9)); \
    prod = prod + (YN(12) * (YN(4) * RCT(1, 10))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(250)))); \
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
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(256)))); \
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
    TM_LD(0, 6, 318); \
    TM_LD(0, 7, 316); \
    TM_LD(0, 8, 336); \
    TM_LD(0, 9, 338); \
    TM_LD(0, 10, 356); \
    TM_LD(0, 11, 358); \
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
    TM_LD(1, 0, 376); \
    TM_LD(1, 1, 378); \
    TM_LD(1, 2, 428); \
    TM_LD(1, 3, 430); \
    TM_LD(1, 4, 442); \
    TM_LD(1, 5, 440); \
    TM_LD(1, 6, 488); \
    TM_LD(1, 7, 490); \
    TM_LD(1, 8, 168); \
    TM_LD(1, 9, 170); \
    TM_LD(1, 10, 186); \
    TM_LD(1, 11, 184); \
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
    TM_WAIT(1); \
    TM_LD(0, 0, 228); \
    TM_LD(0, 1, 230); \
    TM_LD(0, 2, 234); \
    TM_LD(0, 3, 232); \
    TM_LD(0, 4, 238); \
    TM_LD(0, 5, 236); \
    TM_LD(0, 6, 242); \
    TM_LD(0, 7, 240); \
    TM_LD(0, 8, 246); \
    TM_LD(0, 9, 244); \
    TM_LD(0, 10, 250); \
    TM_LD(0, 11, 248); \
    prod = prod + (YN(6) * (YO(24) * RCT(1, 0))); \
    loss = loss + ((YN(8) * YN(7)) * RCT(1, 1)); \
    prod = prod + (YN(2) * (YO(25) * RCT(1, 2))); \
    loss = loss + (YN(8) * RCT(1, 3)); \
    prod = prod + (YN(8) * (YO(18) * RCT(1, 4))); \
    loss = loss + (YO(25) * RCT(1, 5)); \
    prod = prod + (YN(2) * (YO(28) * RCT(1, 6))); \
    loss = loss + (YN(4) * RCT(1, 7)); \
    prod = prod + (YO(29) * RCS(14)); \
    loss = loss + (YN(4) * RCS(15)); \
    prod = prod + (YN(2) * (YO(23) * RCS(18))); \
    loss = loss + (YN(10) * RCS(19)); \
    prod = prod + (YN(8) * ((YO(18) * YN(2)) * RCS(29))); \
    loss = loss + (YO(23) * RCS(28)); \
    prod = prod + (YO(23) * RCS(34)); \
    loss = loss + (YN(8) * RCS(35)); \
    prod = prod + (YO(31) * RCS(36)); \
    loss = loss + (YN(10) * RCS(37)); \
    prod = prod + (YO(34) * RCS(38)); \
    loss = loss + (YN(8) * RCS(39)); \
    prod = prod + (YN(12) * (YO(34) * RCS(53))); \
    loss = loss + (YO(31) * RCS(52)); \
    prod = prod + (YN(12) * (YO(23) * RCS(55))); \
    loss = loss + (YO(31) * RCS(54)); \
    prod = prod + (YO(30) * RCS(62)); \
    loss = loss + (YO(28) * RCS(63)); \
    prod = prod + (YN(12) * (YO(33) * RCS(85))); \
    loss = loss + (YO(30) * RCS(84)); \
    prod = prod + (YN(12) * (YO(32) * RCS(87))); \
    loss = loss + (YO(30) * RCS(86)); \
    prod = prod + (YN(12) * (YO(35) * RCS(89))); \
    loss = loss + (YO(30) * RCS(88)); \
    prod = prod + (YO(35) * RCS(102)); \
    loss = loss + (YN(11) * RCS(103)); \
    prod = prod + (YN(2) * (YO(35) * RCS(108))); \
    loss = loss + (YO(28) * RCS(109)); \
    prod = prod + (YN(2) * (YO(32) * RCS(120))); \
    loss = loss + (YO(28) * RCS(121)); \
    prod = prod + (YN(2) * (YO(36) * RCS(131))); \
    loss = loss + (YO(21) * RCS(130)); \
    prod = prod + (YN(3) * (YO(36) * RCS(132))); \
    loss = loss + (YO(26) * RCS(133)); \
    prod = prod + (YN(12) * (YO(36) * RCS(149))); \
    loss = loss + (YO(38) * RCS(148)); \
    prod = prod + (YO(38) * RCS(151)); \
    loss = loss + (YO(21) * RCS(150)); \
    prod = prod + (YN(1) * (YO(36) * RCS(158))); \
    loss = loss + ((YN(10) * YN(8)) * RCS(159)); \
    prod = prod + (YN(3) * (YO(39) * RCS(164))); \
    loss = loss + ((YO(25) * YN(2)) * RCS(165)); \
    prod = prod + (YO(39) * RCS(175)); \
    loss = loss + (YO(22) * RCS(174)); \
    prod = prod + (YN(2) * (YO(39) * RCS(176))); \
    loss = loss + (YO(16) * RCS(177)); \
    prod = prod + (YN(2) * (YO(38) * RCS(179))); \
    loss = loss + (YO(22) * RCS(178)); \
    prod = prod + (YO(40) * RCS(180)); \
    loss = loss + (YO(18) * RCS(181)); \
    prod = prod + (YO(42) * RCS(208)); \
    loss = loss + (YO(16) * RCS(209)); \
    prod = prod + (YN(12) * ((YO(21) * YO(22)) * RCS(227))); \
    loss = loss + (YO(43) * RCS(226)); \
    prod = prod + (YO(43) * RCS(229)); \
    loss = loss + (YO(37) * RCS(228)); \
    prod = prod + (YN(2) * (YO(48) * RCS(270))); \
    loss = loss + ((YO(16) * YO(16)) * RCS(271)); \
    prod = prod + (YN(2) * (YO(48) * RCS(276))); \
    loss = loss + ((YN(0) * YO(43)) * RCS(277)); \
    prod = prod + (YO(47) * RCS(278)); \
    loss = loss + (YO(38) * RCS(279)); \
    prod = prod + (YN(2) * (YO(47) * RCS(282))); \
    loss = loss + (YO(39) * RCS(283)); \
    rhs1 = rho * Y0S(1) + dt * WM(13) * (prod + extra); \
    rhs2 = -(dt * WM(13) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(13) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(13) - fnew); \
    UC_UPDATE_TAIL(13); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 15); \
    prod = (YN(13) * (YN(2) * RCT(1, 8))); \
    extra = 0.0; \
    loss = (YN(0) * RCT(1, 9)); \
    prod = prod + (YN(2) * (YO(16) * RCT(1, 10))); \
    loss = loss + (YN(13) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 254); \
    TM_LD(1, 1, 252); \
    TM_LD(1, 2, 258); \
    TM_LD(1, 3, 256); \
    TM_LD(1, 4, 262); \
    TM_LD(1, 5, 260); \
    TM_LD(1, 6, 412); \
    TM_LD(1, 7, 414); \
    TM_LD(1, 8, 432); \
    TM_LD(1, 9, 434); \
    TM_LD(1, 10, 172); \
    TM_LD(1, 11, 174); \
    prod = prod + (YO(15) * RCT(0, 0)); \
    loss = loss + RCT(0, 1); \
    prod = prod + (YN(0) * (YO(20) * RCT(0, 2))); \
    loss = loss + (YN(2) * RCT(0, 3)); \
    prod = prod + (YN(11) * (YN(2) * RCT(0, 4))); \
    loss = loss + (YN(4) * RCT(0, 5)); \
    prod = prod + (YN(5) * (YO(20) * RCT(0, 6))); \
    loss = loss + (YN(4) * RCT(0, 7)); \
    prod = prod + (YN(8) * ((YN(2) * YN(2)) * RCT(0, 8))); \
    loss = loss + (YN(3) * RCT(0, 9)); \
    prod = prod + (YN(8) * (YN(0) * RCT(0, 10))); \
    loss = loss + (YN(3) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 176); \
    TM_LD(0, 1, 178); \
    TM_LD(0, 2, 218); \
    TM_LD(0, 3, 216); \
    TM_LD(0, 4, 222); \
    TM_LD(0, 5, 220); \
    TM_LD(0, 6, 226); \
    TM_LD(0, 7, 224); \
    TM_LD(0, 8, 230); \
    TM_LD(0, 9, 228); \
    TM_LD(0, 10, 284); \
    TM_LD(0, 11, 286); \
    prod = prod + (YN(9) * (YN(0) * RCT(1, 0))); \
    loss = loss + (YN(1) * RCT(1, 1)); \
    prod = prod + (YN(8) * ((YN(4) * YN(2)) * RCT(1, 2))); \
    loss = loss + (YN(1) * RCT(1, 3)); \
    prod = prod + (YN(2) * ((YO(21) * YOS(0)) * RCT(1, 4))); \
    loss = loss + (YO(14) * RCT(1, 5)); \
    prod = prod + (YN(2) * ((YO(21) * YOS(0)) * RCT(1, 4))); \
    loss = loss + (YO(14) * RCT(1, 5)); \
    prod = prod + (YN(3) * (YO(21) * RCT(1, 6))); \
    loss = loss + (YN(8) * RCT(1, 7)); \
    prod = prod + (YN(3) * (YO(25) * RCT(1, 8))); \
    loss = loss + (YN(9) * RCT(1, 9)); \
    rhs1 = rho * Y0S(0) + dt * WM(14) * (prod + extra); \
    rhs2 = -(dt * WM(14) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(14) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(14) - fnew); \
    UC_UPDATE_TAIL(14); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 16); \
    prod = (YN(13) * (YN(2) * RCT(1, 10))); \
    extra = 0.0; \
    loss = (YN(0) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 444); \
    TM_LD(1, 1, 446); \
    TM_LD(1, 2, 184); \
    TM_LD(1, 3, 186); \
    TM_LD(1, 4, 200); \
    TM_LD(1, 5, 202); \
    TM_LD(1, 6, 328); \
    TM_LD(1, 7, 330); \
    TM_LD(1, 8, 332); \
    TM_LD(1, 9, 334); \
    TM_LD(1, 10, 340); \
    TM_LD(1, 11, 342); \
    prod = prod + (YN(13) * (YN(4) * RCT(0, 0))); \
    loss = loss + (YN(5) * RCT(0, 1)); \
    prod = prod + (YN(11) * (YN(2) * RCT(0, 2))); \
    loss = loss + (YN(4) * RCT(0, 3)); \
    prod = prod + (YN(8) * ((YN(4) * YN(2)) * RCT(0, 4))); \
    loss = loss + (YN(1) * RCT(0, 5)); \
    prod = prod + (YN(11) * (YN(8) * RCT(0, 6))); \
    loss = loss + (YN(9) * RCT(0, 7)); \
    prod = prod + (YN(14) * RCT(0, 8)); \
    loss = loss + RCT(0, 9); \
    prod = prod + (YN(2) * (YO(17) * RCT(0, 10))); \
    loss = loss + (YN(5) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 344); \
    TM_LD(0, 1, 346); \
    TM_LD(0, 2, 350); \
    TM_LD(0, 3, 348); \
    TM_LD(0, 4, 354); \
    TM_LD(0, 5, 352); \
    TM_LD(0, 6, 358); \
    TM_LD(0, 7, 356); \
    TM_LD(0, 8, 362); \
    TM_LD(0, 9, 360); \
    TM_LD(0, 10, 366); \
    TM_LD(0, 11, 364); \
    prod = prod + (YN(2) * (YO(26) * RCT(1, 0))); \
    loss = loss + (YN(8) * RCT(1, 1)); \
    rhs1 = rho * Y0S(1) + dt * WM(15) * (prod + extra); \
    rhs2 = -(dt * WM(15) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(15) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(15) - fnew); \
    UC_UPDATE_TAIL(15); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 17); \
    prod = (YN(14) * (YN(13) * RCT(1, 2))); \
    extra = (1.0 * (YO(46) * RCS(244))); \
    loss = (YN(2) * RCT(1, 3)); \
    prod = prod + (YN(13) * (YOS(3) * RCT(1, 4))); \
    extra = extra + (1.0 * (YO(46) * RCS(244))); \
    loss = loss + (YN(0) * RCT(1, 5)); \
    prod = prod + (YN(2) * (YO(18) * RCT(1, 6))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(246)))); \
    loss = loss + (YN(0) * RCT(1, 7)); \
    prod = prod + (YN(3) * (YO(18) * RCT(1, 8))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(248)))); \
    loss = loss + (YN(4) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(18) * RCT(1, 10))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(250)))); \
    loss = loss + (YN(6) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 370); \
    TM_LD(1, 1, 368); \
    TM_LD(1, 2, 374); \
    TM_LD(1, 3, 372); \
    TM_LD(1, 4, 382); \
    TM_LD(1, 5, 380); \
    TM_LD(1, 6, 386); \
    TM_LD(1, 7, 384); \
    TM_LD(1, 8, 188); \
    TM_LD(1, 9, 190); \
    TM_LD(1, 10, 196); \
    TM_LD(1, 11, 198); \
    prod = prod + (YO(18) * RCT(0, 0)); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(250)))); \
    loss = loss + (YN(2) * RCT(0, 1)); \
    prod = prod + (YN(0) * (YO(22) * RCT(0, 2))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(250)))); \
    loss = loss + (YN(2) * RCT(0, 3)); \
    prod = prod + (YN(5) * (YO(22) * RCT(0, 4))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(256)))); \
    loss = loss + (YN(4) * RCT(0, 5)); \
    prod = prod + (YN(13) * (YN(10) * RCT(0, 6))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(258)))); \
    loss = loss + (YN(3) * RCT(0, 7)); \
    prod = prod + (YN(2) * (YO(23) * RCT(0, 8))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    loss = loss + (YN(3) * RCT(0, 9)); \
    prod = prod + ((YO(22) * YO(18)) * RCT(0, 10)); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    loss = loss + (YO(16) * RCT(0, 11)); \
    prod = prod + ((YO(22) * YO(18)) * RCT(0, 10)); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(260)))); \
    loss = loss + (YO(16) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 282); \
    TM_LD(0, 1, 280); \
    TM_LD(0, 2, 286); \
    TM_LD(0, 3, 284); \
    TM_LD(0, 4, 290); \
    TM_LD(0, 5, 288); \
    TM_LD(0, 6, 294); \
    TM_LD(0, 7, 292); \
    TM_LD(0, 8, 298); \
    TM_LD(0, 9, 296); \
    TM_LD(0, 10, 302); \
    TM_LD(0, 11, 300); \
    prod = prod + (YN(6) * (YO(22) * RCT(1, 0))); \
    loss = loss + (YN(1) * RCT(1, 1)); \
    prod = prod + (YN(4) * (YO(24) * RCT(1, 2))); \
    loss = loss + (YN(6) * RCT(1, 3)); \
    prod = prod + (YN(2) * (YO(22) * RCT(1, 4))); \
    loss = loss + RCT(1, 5); \
    prod = prod + (YN(0) * (YO(21) * RCT(1, 6))); \
    loss = loss + RCT(1, 7); \
    prod = prod + (YO(30) * RCS(64)); \
    loss = loss + (YN(5) * RCS(65)); \
    prod = prod + (YO(33) * RCS(97)); \
    loss = loss + (YN(4) * RCS(96)); \
    prod = prod + (YN(2) * (YO(35) * RCS(110))); \
    loss = loss + (YN(5) * RCS(111)); \
    prod = prod + (YN(2) * (YO(32) * RCS(118))); \
    loss = loss + (YN(5) * RCS(119)); \
    prod = prod + (YN(3) * (YO(36) * RCS(128))); \
    loss = loss + (YN(8) * RCS(129)); \
    prod = prod + (YN(2) * (YO(39) * RCS(176))); \
    loss = loss + (YN(13) * RCS(177)); \
    prod = prod + (YO(42) * RCS(208)); \
    loss = loss + (YN(13) * RCS(209)); \
    prod = prod + (YN(2) * (YO(43) * RCS(220))); \
    loss = loss + (YO(22) * RCS(221)); \
    prod = prod + (YO(45) * RCS(232)); \
    loss = loss + (YO(36) * RCS(233)); \
    prod = prod + (YO(48) * RCS(264)); \
    loss = loss + (YO(39) * RCS(265)); \
    prod = prod + (YN(2) * (YO(48) * RCS(270))); \
    loss = loss + ((YO(16) * YN(13)) * RCS(271)); \
    prod = prod + (YN(2) * (YO(48) * RCS(270))); \
    loss = loss + ((YO(16) * YN(13)) * RCS(271)); \
    prod = prod + (YN(2) * (YO(48) * RCS(274))); \
    loss = loss + ((YN(0) * YO(38)) * RCS(275)); \
    prod = prod + (YN(2) * (YO(47) * RCS(280))); \
    loss = loss + (YO(18) * RCS(281)); \
    prod = prod + (YN(2) * (YO(47) * RCS(284))); \
    loss = loss + ((YN(0) * YO(22)) * RCS(285)); \
    rhs1 = rho * Y0S(0) + dt * WM(16) * (prod + extra); \
    rhs2 = -(dt * WM(16) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(16) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(16) - fnew); \
    UC_UPDATE_TAIL(16); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 18); \
    prod = (YN(13) * (YN(6) * RCT(1, 8))); \
    extra = 0.0; \
    loss = (YN(4) * RCT(1, 9)); \
    prod = prod + (YN(13) * (YN(1) * RCT(1, 10))); \
    loss = loss + (YN(3) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 506); \
    TM_LD(1, 1, 504); \
    TM_LD(1, 2, 204); \
    TM_LD(1, 3, 206); \
    TM_LD(1, 4, 304); \
    TM_LD(1, 5, 306); \
    TM_LD(1, 6, 308); \
    TM_LD(1, 7, 310); \
    TM_LD(1, 8, 312); \
    TM_LD(1, 9, 314); \
    TM_LD(1, 10, 316); \
    TM_LD(1, 11, 318); \
    prod = prod + (YN(11) * (YN(0) * RCT(0, 0))); \
    loss = loss + (YN(2) * RCT(0, 1)); \
    prod = prod + (YN(15) * (YN(5) * RCT(0, 2))); \
    loss = loss + (YN(2) * RCT(0, 3)); \
    prod = prod + (YN(11) * (YN(5) * RCT(0, 4))); \
    loss = loss + (YN(4) * RCT(0, 5)); \
    prod = prod + (YN(11) * (YN(4) * RCT(0, 6))); \
    loss = loss + (YN(3) * RCT(0, 7)); \
    prod = prod + (YN(11) * (YN(6) * RCT(0, 8))); \
    loss = loss + (YN(1) * RCT(0, 9)); \
    prod = prod + (YN(11) * (YN(2) * RCT(0, 10))); \
    loss = loss + RCT(0, 11); \
    TM_WAIT(1); \
    TM_LD(0, 0, 320); \
    TM_LD(0, 1, 322); \
    TM_LD(0, 2, 324); \
    TM_LD(0, 3, 326); \
    TM_LD(0, 4, 330); \
    TM_LD(0, 5, 328); \
    TM_LD(0, 6, 334); \
    TM_LD(0, 7, 332); \
    TM_LD(0, 8, 338); \
    TM_LD(0, 9, 336); \
    TM_LD(0, 10, 342); \
    TM_LD(0, 11, 340); \
    prod = prod + (YO(28) * RCT(1, 0)); \
    loss = loss + RCT(1, 1); \
    prod = prod + (YN(4) * (YO(29) * RCS(2))); \
    loss = loss + (YN(5) * RCS(3)); \
    prod = prod + (YN(2) * (YO(29) * RCS(6))); \
    loss = loss + (YN(0) * RCS(7)); \
    rhs1 = rho * Y0S(1) + dt * WM(17) * (prod + extra); \
    rhs2 = -(dt * WM(17) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(17) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(17) - fnew); \
    UC_UPDATE_TAIL(17); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 19); \
    prod = (YN(13) * (YOS(3) * RCT(1, 2))); \
    extra = (1.0 * (YO(46) * RCS(244))); \
    loss = (YN(2) * RCT(1, 3)); \
    prod = prod + (YN(2) * (YO(19) * RCT(1, 4))); \
    extra = extra + (1.0 * (YN(2) * (YO(46) * RCS(246)))); \
    loss = loss + (YN(0) * RCT(1, 5)); \
    prod = prod + (YN(3) * (YO(19) * RCT(1, 6))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(258)))); \
    loss = loss + (YN(4) * RCT(1, 7)); \
    prod = prod + (YN(4) * (YO(19) * RCT(1, 8))); \
    loss = loss + (YN(5) * RCT(1, 9)); \
    prod = prod + (YN(13) * (YO(19) * RCT(1, 10))); \
    loss = loss + (YN(12) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 346); \
    TM_LD(1, 1, 344); \
    TM_LD(1, 2, 364); \
    TM_LD(1, 3, 366); \
    TM_LD(1, 4, 440); \
    TM_LD(1, 5, 442); \
    TM_LD(1, 6, 212); \
    TM_LD(1, 7, 214); \
    TM_LD(1, 8, 306); \
    TM_LD(1, 9, 304); \
    TM_LD(1, 10, 310); \
    TM_LD(1, 11, 308); \
    prod = prod + (YO(19) * RCT(0, 0)); \
    loss = loss + (YN(2) * RCT(0, 1)); \
    prod = prod + (YN(6) * (YO(19) * RCT(0, 2))); \
    loss = loss + (YN(7) * RCT(0, 3)); \
    prod = prod + (YN(16) * (YN(0) * RCT(0, 4))); \
    loss = loss + (YN(2) * RCT(0, 5)); \
    prod = prod + (YN(16) * (YN(4) * RCT(0, 6))); \
    loss = loss + (YN(3) * RCT(0, 7)); \
    prod = prod + (YN(13) * (YN(11) * RCT(0, 8))); \
    loss = loss + (YN(3) * RCT(0, 9)); \
    prod = prod + (YN(16) * (YN(6) * RCT(0, 10))); \
    loss = loss + (YN(1) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 314); \
    TM_LD(0, 1, 312); \
    TM_LD(0, 2, 318); \
    TM_LD(0, 3, 316); \
    TM_LD(0, 4, 322); \
    TM_LD(0, 5, 320); \
    TM_LD(0, 6, 326); \
    TM_LD(0, 7, 324); \
    TM_LD(0, 8, 232); \
    TM_LD(0, 9, 234); \
    TM_LD(0, 10, 240); \
    TM_LD(0, 11, 242); \
    prod = prod + (YN(16) * (YN(2) * RCT(1, 0))); \
    loss = loss + RCT(1, 1); \
    prod = prod + (YN(16) * (YOS(4) * RCT(1, 2))); \
    loss = loss + (YO(22) * RCT(1, 3)); \
    prod = prod + (YN(13) * (YO(25) * RCT(1, 4))); \
    loss = loss + (YN(8) * RCT(1, 5)); \
    prod = prod + (YN(13) * (YO(23) * RCS(28))); \
    loss = loss + ((YN(8) * YN(2)) * RCS(29)); \
    prod = prod + (YN(4) * (YO(35) * RCS(99))); \
    loss = loss + (YN(6) * RCS(98)); \
    prod = prod + (YN(8) * (YO(35) * RCS(106))); \
    loss = loss + (YN(9) * RCS(107)); \
    prod = prod + (YN(3) * (YO(39) * RCS(160))); \
    loss = loss + (YN(10) * RCS(161)); \
    prod = prod + (YO(40) * RCS(180)); \
    loss = loss + (YN(13) * RCS(181)); \
    prod = prod + (YN(2) * (YO(46) * RCS(252))); \
    loss = loss + ((YN(0) * YO(48)) * RCS(253)); \
    prod = prod + (YN(4) * (YO(46) * RCS(254))); \
    loss = loss + ((YN(5) * YO(48)) * RCS(255)); \
    prod = prod + (YO(48) * RCS(262)); \
    loss = loss + (YO(38) * RCS(263)); \
    prod = prod + (YN(2) * (YO(48) * RCS(272))); \
    loss = loss + (YO(39) * RCS(273)); \
    prod = prod + (YN(2) * (YO(47) * RCS(280))); \
    loss = loss + (YN(16) * RCS(281)); \
    rhs1 = rho * Y0S(0) + dt * WM(18) * (prod + extra); \
    rhs2 = -(dt * WM(18) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(18) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(18) - fnew); \
    UC_UPDATE_TAIL(18); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 20); \
    prod = (YN(13) * (YOS(3) * RCT(1, 6))); \
    extra = 0.0; \
    loss = RCT(1, 7); \
    prod = prod + (YN(18) * (YN(0) * RCT(1, 8))); \
    loss = loss + (YN(2) * RCT(1, 9)); \
    prod = prod + (YN(18) * (YN(4) * RCT(1, 10))); \
    loss = loss + (YN(3) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 266); \
    TM_LD(1, 1, 264); \
    TM_LD(1, 2, 270); \
    TM_LD(1, 3, 268); \
    TM_LD(1, 4, 274); \
    TM_LD(1, 5, 272); \
    TM_LD(1, 6, 278); \
    TM_LD(1, 7, 276); \
    TM_LD(1, 8, 468); \
    TM_LD(1, 9, 470); \
    TM_LD(1, 10, 476); \
    TM_LD(1, 11, 478); \
    prod = prod + (YN(18) * (YN(5) * RCT(0, 0))); \
    loss = loss + (YN(4) * RCT(0, 1)); \
    prod = prod + (YN(18) * (YN(12) * RCT(0, 2))); \
    loss = loss + (YN(13) * RCT(0, 3)); \
    prod = prod + (YN(18) * (YN(2) * RCT(0, 4))); \
    loss = loss + RCT(0, 5); \
    prod = prod + (YN(18) * (YN(7) * RCT(0, 6))); \
    loss = loss + (YN(6) * RCT(0, 7)); \
    rhs1 = rho * Y0S(1) + dt * WM(19) * (prod + extra); \
    rhs2 = -(dt * WM(19) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(19) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(19) - fnew); \
    UC_UPDATE_TAIL(19); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 21); \
    prod = (YN(14) * (YN(2) * RCT(0, 8))); \
    extra = 0.0; \
    loss = (YN(0) * RCT(0, 9)); \
    prod = prod + (YN(14) * (YN(4) * RCT(0, 10))); \
    loss = loss + (YN(5) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 260); \
    TM_LD(0, 1, 262); \
    TM_LD(0, 2, 384); \
    TM_LD(0, 3, 386); \
    TM_LD(0, 4, 388); \
    TM_LD(0, 5, 390); \
    TM_LD(0, 6, 392); \
    TM_LD(0, 7, 394); \
    TM_LD(0, 8, 404); \
    TM_LD(0, 9, 406); \
    TM_LD(0, 10, 410); \
    TM_LD(0, 11, 408); \
    prod = prod + (YN(8) * (YN(2) * RCT(1, 0))); \
    loss = loss + (YN(3) * RCT(1, 1)); \
    prod = prod + (YN(10) * (YN(3) * RCT(1, 2))); \
    loss = loss + (YN(1) * RCT(1, 3)); \
    prod = prod + (YN(11) * (YN(2) * RCT(1, 4))); \
    loss = loss + (YN(5) * RCT(1, 5)); \
    prod = prod + (YN(10) * (YN(8) * RCT(1, 6))); \
    loss = loss + (YN(9) * RCT(1, 7)); \
    prod = prod + (YN(3) * (YO(27) * RCT(1, 8))); \
    loss = loss + (YN(8) * RCT(1, 9)); \
    prod = prod + (YN(1) * (YO(27) * RCT(1, 10))); \
    loss = loss + (YN(9) * RCT(1, 11)); \
    rhs1 = rho * Y0S(0) + dt * WM(20) * (prod + extra); \
    rhs2 = -(dt * WM(20) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(20) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(20) - fnew); \
    UC_UPDATE_TAIL(20); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 22); \
    TM_WAIT(0); \
    TM_LD(1, 0, 414); \
    TM_LD(1, 1, 412); \
    TM_LD(1, 2, 418); \
    TM_LD(1, 3, 416); \
    TM_LD(1, 4, 422); \
    TM_LD(1, 5, 420); \
    TM_LD(1, 6, 426); \
    TM_LD(1, 7, 424); \
    TM_LD(1, 8, 348); \
    TM_LD(1, 9, 350); \
    TM_LD(1, 10, 352); \
    TM_LD(1, 11, 354); \
    prod = (YN(14) * (YOS(5) * RCT(0, 0))); \
    extra = 0.0; \
    loss = ((YN(2) * YN(2)) * RCT(0, 1)); \
    prod = prod + (YN(16) * RCT(0, 2)); \
    loss = loss + (YN(0) * RCT(0, 3)); \
    prod = prod + (YN(2) * (YO(22) * RCT(0, 4))); \
    loss = loss + (YN(0) * RCT(0, 5)); \
    prod = prod + (YO(22) * RCT(0, 6)); \
    loss = loss + (YN(2) * RCT(0, 7)); \
    prod = prod + (YN(1) * (YO(22) * RCT(0, 8))); \
    loss = loss + (YN(6) * RCT(0, 9)); \
    prod = prod + (YN(2) * (YO(26) * RCT(0, 10))); \
    loss = loss + (YN(3) * RCT(0, 11)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 364); \
    TM_LD(0, 1, 366); \
    TM_LD(0, 2, 368); \
    TM_LD(0, 3, 370); \
    TM_LD(0, 4, 380); \
    TM_LD(0, 5, 382); \
    TM_LD(0, 6, 390); \
    TM_LD(0, 7, 388); \
    TM_LD(0, 8, 394); \
    TM_LD(0, 9, 392); \
    TM_LD(0, 10, 398); \
    TM_LD(0, 11, 396); \
    prod = prod + (YN(14) * (YN(8) * RCT(1, 0))); \
    loss = loss + (YN(3) * RCT(1, 1)); \
    prod = prod + (YN(11) * (YN(8) * RCT(1, 2))); \
    loss = loss + (YN(1) * RCT(1, 3)); \
    prod = prod + (YN(2) * (YO(25) * RCT(1, 4))); \
    loss = loss + (YN(4) * RCT(1, 5)); \
    prod = prod + (YN(5) * (YO(27) * RCT(1, 6))); \
    loss = loss + (YN(4) * RCT(1, 7)); \
    prod = prod + (YN(2) * (YO(36) * RCS(131))); \
    loss = loss + (YN(13) * RCS(130)); \
    prod = prod + (YO(38) * RCS(151)); \
    loss = loss + (YN(13) * RCS(150)); \
    prod = prod + (YO(43) * RCS(214)); \
    loss = loss + ((YO(22) * YN(2)) * RCS(215)); \
    prod = prod + (YN(2) * (YO(43) * RCS(222))); \
    loss = loss + ((YN(0) * YO(22)) * RCS(223)); \
    prod = prod + (YN(13) * (YO(43) * RCS(226))); \
    loss = loss + ((YN(12) * YO(22)) * RCS(227)); \
    prod = prod + (YO(45) * RCS(230)); \
    loss = loss + (YO(39) * RCS(231)); \
    prod = prod + (YN(1) * (YO(45) * RCS(236))); \
    loss = loss + ((YO(38) * YN(6)) * RCS(237)); \
    prod = prod + (YN(6) * (YO(45) * RCS(240))); \
    loss = loss + ((YO(38) * YN(7)) * RCS(241)); \
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
    TM_LD(1, 0, 402); \
    TM_LD(1, 1, 400); \
    TM_LD(1, 2, 406); \
    TM_LD(1, 3, 404); \
    TM_LD(1, 4, 360); \
    TM_LD(1, 5, 362); \
    TM_LD(1, 6, 372); \
    TM_LD(1, 7, 374); \
    TM_LD(1, 8, 378); \
    TM_LD(1, 9, 376); \
    TM_LD(1, 10, 420); \
    TM_LD(1, 11, 422); \
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
    TM_LD(0, 0, 430); \
    TM_LD(0, 1, 428); \
    TM_LD(0, 2, 434); \
    TM_LD(0, 3, 432); \
    TM_LD(0, 4, 438); \
    TM_LD(0, 5, 436); \
    TM_LD(0, 6, 442); \
    TM_LD(0, 7, 440); \
    TM_LD(0, 8, 510); \
    TM_LD(0, 9, 508); \
    TM_LD(0, 10, 408); \
    TM_LD(0, 11, 410); \
    prod = prod + (YN(3) * (YO(23) * RCT(1, 0))); \
    loss = loss + (YN(1) * RCT(1, 1)); \
    prod = prod + (YN(21) * (YN(6) * RCT(1, 2))); \
    loss = loss + (YN(1) * RCT(1, 3)); \
    prod = prod + (YN(6) * (YO(37) * RCS(156))); \
    loss = loss + ((YN(4) * YN(8)) * RCS(157)); \
    prod = prod + (YN(6) * (YO(38) * RCS(172))); \
    loss = loss + ((YN(4) * YN(11)) * RCS(173)); \
    prod = prod + (YO(39) * RCS(175)); \
    loss = loss + (YN(13) * RCS(174)); \
    prod = prod + (YN(2) * (YO(38) * RCS(179))); \
    loss = loss + (YN(13) * RCS(178)); \
    prod = prod + (YO(43) * RCS(214)); \
    loss = loss + ((YN(21) * YN(2)) * RCS(215)); \
    prod = prod + (YO(43) * RCS(216)); \
    loss = loss + (YO(22) * RCS(217)); \
    prod = prod + (YO(43) * RCS(216)); \
    loss = loss + (YO(22) * RCS(217)); \
    prod = prod + (YO(43) * RCS(219)); \
    loss = loss + (YO(22) * RCS(218)); \
    prod = prod + (YO(43) * RCS(219)); \
    loss = loss + (YO(22) * RCS(218)); \
    prod = prod + (YN(2) * (YO(43) * RCS(220))); \
    loss = loss + (YN(16) * RCS(221)); \
    prod = prod + (YN(2) * (YO(43) * RCS(222))); \
    loss = loss + ((YN(0) * YN(21)) * RCS(223)); \
    prod = prod + (YN(13) * (YO(43) * RCS(226))); \
    loss = loss + ((YN(12) * YN(21)) * RCS(227)); \
    prod = prod + (YO(45) * RCS(234)); \
    loss = loss + (YO(38) * RCS(235)); \
    prod = prod + (YN(1) * (YO(45) * RCS(238))); \
    loss = loss + ((YO(36) * YN(6)) * RCS(239)); \
    prod = prod + (YN(6) * (YO(45) * RCS(242))); \
    loss = loss + ((YO(36) * YN(7)) * RCS(243)); \
    prod = prod + (YN(4) * (YO(48) * RCS(266))); \
    loss = loss + ((YN(5) * YO(39)) * RCS(267)); \
    prod = prod + (YN(2) * (YO(48) * RCS(268))); \
    loss = loss + ((YN(0) * YO(39)) * RCS(269)); \
    prod = prod + (YN(2) * (YO(47) * RCS(284))); \
    loss = loss + ((YN(0) * YN(16)) * RCS(285)); \
    rhs1 = rho * Y0S(0) + dt * WM(22) * (prod + extra); \
    rhs2 = -(dt * WM(22) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(22) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(22) - fnew); \
    UC_UPDATE_TAIL(22); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 24); \
    prod = (YN(16) * (YN(3) * RCT(1, 4))); \
    extra = 0.0; \
    loss = (YN(2) * RCT(1, 5)); \
    prod = prod + (YN(22) * (YN(1) * RCT(1, 1))); \
    loss = loss + (YN(3) * RCT(1, 0)); \
    prod = prod + (YN(2) * (YO(25) * RCS(17))); \
    loss = loss + RCS(16); \
    prod = prod + (YN(13) * (YN(10) * RCS(19))); \
    loss = loss + (YN(2) * RCS(18)); \
    prod = prod + (YN(0) * (YO(25) * RCS(21))); \
    loss = loss + (YN(2) * RCS(20)); \
    prod = prod + (YN(11) * (YN(10) * RCS(23))); \
    loss = loss + (YN(3) * RCS(22)); \
    prod = prod + (YN(5) * (YO(25) * RCS(25))); \
    loss = loss + (YN(4) * RCS(24)); \
    prod = prod + (YN(11) * ((YN(8) * YN(4)) * RCS(27))); \
    loss = loss + (YN(1) * RCS(26)); \
    prod = prod + (YN(18) * ((YN(8) * YN(2)) * RCS(29))); \
    loss = loss + (YN(13) * RCS(28)); \
    prod = prod + (YN(11) * ((YN(10) * YN(4)) * RCS(31))); \
    loss = loss + (YN(6) * RCS(30)); \
    prod = prod + (YN(1) * (YO(31) * RCS(33))); \
    loss = loss + (YN(6) * RCS(32)); \
    prod = prod + (YN(13) * (YN(8) * RCS(35))); \
    loss = loss + RCS(34); \
    prod = prod + (YN(4) * (YO(31) * RCS(42))); \
    loss = loss + (YN(5) * RCS(43)); \
    prod = prod + (YN(3) * (YO(31) * RCS(46))); \
    loss = loss + (YN(4) * RCS(47)); \
    prod = prod + (YN(2) * (YO(31) * RCS(50))); \
    loss = loss + (YN(0) * RCS(51)); \
    prod = prod + (YN(13) * (YO(31) * RCS(54))); \
    loss = loss + (YN(12) * RCS(55)); \
    prod = prod + (YN(6) * (YO(31) * RCS(58))); \
    loss = loss + (YN(7) * RCS(59)); \
    rhs1 = rho * Y0S(1) + dt * WM(23) * (prod + extra); \
    rhs2 = -(dt * WM(23) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(23) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(23) - fnew); \
    UC_UPDATE_TAIL(23); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 25); \
    prod = (YN(16) * (YN(6) * RCT(1, 6))); \
    extra = 0.0; \
    loss = (YN(4) * RCT(1, 7)); \
    prod = prod + (YN(13) * ((YN(8) * YN(7)) * RCT(1, 8))); \
    loss = loss + (YN(6) * RCT(1, 9)); \
    rhs1 = rho * Y0S(0) + dt * WM(24) * (prod + extra); \
    rhs2 = -(dt * WM(24) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(24) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(24) - fnew); \
    UC_UPDATE_TAIL(24); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 26); \
    prod = (YN(21) * (YN(4) * RCT(1, 10))); \
    extra = 0.0; \
    loss = (YN(2) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 446); \
    TM_LD(1, 1, 444); \
    TM_LD(1, 2, 450); \
    TM_LD(1, 3, 448); \
    TM_LD(1, 4, 454); \
    TM_LD(1, 5, 452); \
    TM_LD(1, 6, 458); \
    TM_LD(1, 7, 456); \
    TM_LD(1, 8, 462); \
    TM_LD(1, 9, 460); \
    TM_LD(1, 10, 464); \
    TM_LD(1, 11, 466); \
    prod = prod + (YN(13) * (YN(8) * RCT(0, 0))); \
    loss = loss + (YN(2) * RCT(0, 1)); \
    prod = prod + (YN(14) * (YN(9) * RCT(0, 2))); \
    loss = loss + (YN(3) * RCT(0, 3)); \
    prod = prod + (YN(4) * (YO(26) * RCT(0, 4))); \
    loss = loss + (YN(3) * RCT(0, 5)); \
    prod = prod + (YN(18) * (YN(8) * RCT(0, 6))); \
    loss = loss + (YN(13) * RCT(0, 7)); \
    prod = prod + (YN(8) * (YO(28) * RCT(0, 8))); \
    loss = loss + (YN(4) * RCT(0, 9)); \
    prod = prod + (YN(23) * RCS(16)); \
    loss = loss + (YN(2) * RCS(17)); \
    prod = prod + (YN(23) * (YN(2) * RCS(20))); \
    loss = loss + (YN(0) * RCS(21)); \
    prod = prod + (YN(23) * (YN(4) * RCS(24))); \
    loss = loss + (YN(5) * RCS(25)); \
    prod = prod + (YN(1) * (YO(37) * RCS(140))); \
    loss = loss + (YN(10) * RCS(141)); \
    prod = prod + (YN(3) * (YO(39) * RCS(164))); \
    loss = loss + ((YN(13) * YN(2)) * RCS(165)); \
    rhs1 = rho * Y0S(1) + dt * WM(25) * (prod + extra); \
    rhs2 = -(dt * WM(25) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(25) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(25) - fnew); \
    UC_UPDATE_TAIL(25); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 27); \
    prod = (YN(21) * (YN(3) * RCT(0, 10))); \
    extra = 0.0; \
    loss = (YN(2) * RCT(0, 11)); \
    prod = prod + (YN(25) * (YN(3) * RCT(0, 5))); \
    loss = loss + (YN(4) * RCT(0, 4)); \
    TM_WAIT(1); \
    TM_LD(0, 0, 472); \
    TM_LD(0, 1, 474); \
    TM_LD(0, 2, 424); \
    TM_LD(0, 3, 426); \
    TM_LD(0, 4, 466); \
    TM_LD(0, 5, 464); \
    TM_LD(0, 6, 470); \
    TM_LD(0, 7, 468); \
    TM_LD(0, 8, 478); \
    TM_LD(0, 9, 476); \
    TM_LD(0, 10, 482); \
    TM_LD(0, 11, 480); \
    prod = prod + (YN(15) * (YN(8) * RCT(1, 0))); \
    loss = loss + (YN(2) * RCT(1, 1)); \
    prod = prod + (YN(10) * ((YN(8) * YN(2)) * RCT(1, 2))); \
    loss = loss + (YN(4) * RCT(1, 3)); \
    prod = prod + (YN(8) * ((YOS(6) * YN(2)) * RCT(1, 4))); \
    loss = loss + (YN(3) * RCT(1, 5)); \
    prod = prod + (YN(8) * ((YOS(6) * YN(4)) * RCT(1, 6))); \
    loss = loss + (YN(1) * RCT(1, 7)); \
    prod = prod + (YN(9) * ((YN(8) * YN(2)) * RCT(1, 8))); \
    loss = loss + (YN(1) * RCT(1, 9)); \
    prod = prod + (YN(4) * (YO(27) * RCT(1, 10))); \
    loss = loss + (YN(2) * RCT(1, 11)); \
    TM_WAIT(0); \
    TM_LD(1, 0, 486); \
    TM_LD(1, 1, 484); \
    TM_LD(1, 2, 490); \
    TM_LD(1, 3, 488); \
    TM_LD(1, 4, 494); \
    TM_LD(1, 5, 492); \
    TM_LD(1, 6, 498); \
    TM_LD(1, 7, 496); \
    TM_LD(1, 8, 502); \
    TM_LD(1, 9, 500); \
    TM_LD(1, 10, 504); \
    TM_LD(1, 11, 506); \
    prod = prod + (YN(1) * (YO(27) * RCT(0, 0))); \
    loss = loss + (YN(3) * RCT(0, 1)); \
    prod = prod + (YN(3) * (YO(36) * RCS(132))); \
    loss = loss + (YN(13) * RCS(133)); \
    rhs1 = rho * Y0S(0) + dt * WM(26) * (prod + extra); \
    rhs2 = -(dt * WM(26) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(26) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(26) - fnew); \
    UC_UPDATE_TAIL(26); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 28); \
    prod = (YN(21) * (YN(4) * RCT(0, 2))); \
    extra = 0.0; \
    loss = (YN(5) * RCT(0, 3)); \
    prod = prod + (YN(26) * (YN(2) * RCT(0, 4))); \
    loss = loss + (YN(4) * RCT(0, 5)); \
    prod = prod + (YN(20) * (YN(8) * RCT(0, 6))); \
    loss = loss + (YN(3) * RCT(0, 7)); \
    prod = prod + (YN(26) * (YN(3) * RCT(0, 1))); \
    loss = loss + (YN(1) * RCT(0, 0)); \
    prod = prod + (YN(20) * (YN(9) * RCT(0, 8))); \
    loss = loss + (YN(1) * RCT(0, 9)); \
    prod = prod + (YN(10) * (YN(8) * RCT(0, 10))); \
    loss = loss + (YN(1) * RCT(0, 11)); \
    rhs1 = rho * Y0S(1) + dt * WM(27) * (prod + extra); \
    rhs2 = -(dt * WM(27) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(27) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(27) - fnew); \
    UC_UPDATE_TAIL(27); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 29); \
    TM_WAIT(1); \
    TM_LD(0, 0, 508); \
    TM_LD(0, 1, 510); \
    prod = (YN(11) * (YN(0) * RCT(1, 0))); \
    extra = 0.0; \
    loss = (YN(2) * RCT(1, 1)); \
    prod = prod + (YN(13) * (YN(4) * RCT(1, 2))); \
    loss = loss + (YN(2) * RCT(1, 3)); \
    prod = prod + (YN(11) * (YN(5) * RCT(1, 4))); \
    loss = loss + (YN(4) * RCT(1, 5)); \
    prod = prod + (YN(11) * (YN(6) * RCT(1, 6))); \
    loss = loss + (YN(1) * RCT(1, 7)); \
    prod = prod + (YN(11) * (YN(2) * RCT(1, 8))); \
    loss = loss + RCT(1, 9); \
    prod = prod + (YN(17) * RCT(1, 10)); \
    loss = loss + RCT(1, 11); \
    TM_WAIT(0); \
    prod = prod + (YN(25) * (YN(4) * RCT(0, 0))); \
    loss = loss + (YN(8) * RCT(0, 1)); \
    prod = prod + (YN(4) * (YO(29) * RCS(0))); \
    loss = loss + (YN(5) * RCS(1)); \
    prod = prod + (YN(2) * (YO(29) * RCS(4))); \
    loss = loss + (YN(0) * RCS(5)); \
    prod = prod + (YN(3) * (YO(29) * RCS(8))); \
    loss = loss + (YN(4) * RCS(9)); \
    prod = prod + (YN(6) * (YO(29) * RCS(10))); \
    loss = loss + (YN(7) * RCS(11)); \
    prod = prod + (YN(1) * (YO(29) * RCS(12))); \
    loss = loss + (YN(6) * RCS(13)); \
    prod = prod + (YO(30) * RCS(62)); \
    loss = loss + (YN(13) * RCS(63)); \
    prod = prod + (YN(2) * (YO(35) * RCS(108))); \
    loss = loss + (YN(13) * RCS(109)); \
    prod = prod + (YN(2) * (YO(32) * RCS(120))); \
    loss = loss + (YN(13) * RCS(121)); \
    rhs1 = rho * Y0S(0) + dt * WM(28) * (prod + extra); \
    rhs2 = -(dt * WM(28) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(28) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(28) - fnew); \
    UC_UPDATE_TAIL(28); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 30); \
    prod = (YN(28) * (YN(5) * RCS(1))); \
    extra = 0.0; \
    loss = (YN(4) * RCS(0)); \
    prod = prod + (YN(17) * (YN(5) * RCS(3))); \
    loss = loss + (YN(4) * RCS(2)); \
    prod = prod + (YN(28) * (YN(0) * RCS(5))); \
    loss = loss + (YN(2) * RCS(4)); \
    prod = prod + (YN(17) * (YN(0) * RCS(7))); \
    loss = loss + (YN(2) * RCS(6)); \
    prod = prod + (YN(28) * (YN(4) * RCS(9))); \
    loss = loss + (YN(3) * RCS(8)); \
    prod = prod + (YN(28) * (YN(7) * RCS(11))); \
    loss = loss + (YN(6) * RCS(10)); \
    prod = prod + (YN(28) * (YN(6) * RCS(13))); \
    loss = loss + (YN(1) * RCS(12)); \
    prod = prod + (YN(13) * (YN(4) * RCS(15))); \
    loss = loss + RCS(14); \
    rhs1 = rho * Y0S(1) + dt * WM(29) * (prod + extra); \
    rhs2 = -(dt * WM(29) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(29) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(29) - fnew); \
    UC_UPDATE_TAIL(29); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 31); \
    prod = (YN(28) * (YN(13) * RCS(63))); \
    extra = 0.0; \
    loss = RCS(62); \
    prod = prod + (YN(16) * (YN(5) * RCS(65))); \
    loss = loss + RCS(64); \
    prod = prod + (YN(5) * (YO(33) * RCS(67))); \
    loss = loss + (YN(4) * RCS(66)); \
    prod = prod + (YN(5) * (YO(32) * RCS(69))); \
    loss = loss + (YN(4) * RCS(68)); \
    prod = prod + (YN(5) * (YO(35) * RCS(71))); \
    loss = loss + (YN(4) * RCS(70)); \
    prod = prod + (YN(0) * (YO(33) * RCS(73))); \
    loss = loss + (YN(2) * RCS(72)); \
    prod = prod + (YN(0) * (YO(32) * RCS(75))); \
    loss = loss + (YN(2) * RCS(74)); \
    prod = prod + (YN(0) * (YO(35) * RCS(77))); \
    loss = loss + (YN(2) * RCS(76)); \
    prod = prod + (YN(4) * (YO(33) * RCS(79))); \
    loss = loss + (YN(3) * RCS(78)); \
    prod = prod + (YN(4) * (YO(32) * RCS(81))); \
    loss = loss + (YN(3) * RCS(80)); \
    prod = prod + (YN(4) * (YO(35) * RCS(83))); \
    loss = loss + (YN(3) * RCS(82)); \
    prod = prod + (YN(12) * (YO(33) * RCS(85))); \
    loss = loss + (YN(13) * RCS(84)); \
    prod = prod + (YN(12) * (YO(32) * RCS(87))); \
    loss = loss + (YN(13) * RCS(86)); \
    prod = prod + (YN(12) * (YO(35) * RCS(89))); \
    loss = loss + (YN(13) * RCS(88)); \
    prod = prod + (YN(7) * (YO(32) * RCS(91))); \
    loss = loss + (YN(6) * RCS(90)); \
    prod = prod + (YN(7) * (YO(33) * RCS(93))); \
    loss = loss + (YN(6) * RCS(92)); \
    prod = prod + (YN(7) * (YO(35) * RCS(95))); \
    loss = loss + (YN(6) * RCS(94)); \
    rhs1 = rho * Y0S(0) + dt * WM(30) * (prod + extra); \
    rhs2 = -(dt * WM(30) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(30) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(30) - fnew); \
    UC_UPDATE_TAIL(30); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 32); \
    prod = (YN(23) * (YN(6) * RCS(32))); \
    extra = 0.0; \
    loss = (YN(1) * RCS(33)); \
    prod = prod + (YN(13) * (YN(10) * RCS(37))); \
    loss = loss + RCS(36); \
    prod = prod + (YN(5) * (YO(34) * RCS(41))); \
    loss = loss + (YN(4) * RCS(40)); \
    prod = prod + (YN(23) * (YN(5) * RCS(43))); \
    loss = loss + (YN(4) * RCS(42)); \
    prod = prod + (YN(4) * (YO(34) * RCS(45))); \
    loss = loss + (YN(3) * RCS(44)); \
    prod = prod + (YN(23) * (YN(4) * RCS(47))); \
    loss = loss + (YN(3) * RCS(46)); \
    prod = prod + (YN(0) * (YO(34) * RCS(49))); \
    loss = loss + (YN(2) * RCS(48)); \
    prod = prod + (YN(23) * (YN(0) * RCS(51))); \
    loss = loss + (YN(2) * RCS(50)); \
    prod = prod + (YN(12) * (YO(34) * RCS(53))); \
    loss = loss + (YN(13) * RCS(52)); \
    prod = prod + (YN(23) * (YN(12) * RCS(55))); \
    loss = loss + (YN(13) * RCS(54)); \
    prod = prod + (YN(7) * (YO(34) * RCS(57))); \
    loss = loss + (YN(6) * RCS(56)); \
    prod = prod + (YN(23) * (YN(7) * RCS(59))); \
    loss = loss + (YN(6) * RCS(58)); \
    prod = prod + (YN(6) * (YO(34) * RCS(61))); \
    loss = loss + (YN(1) * RCS(60)); \
    prod = prod + (YO(35) * RCS(100)); \
    loss = loss + (YN(2) * RCS(101)); \
    prod = prod + (YN(1) * (YO(35) * RCS(104))); \
    loss = loss + (YN(6) * RCS(105)); \
    prod = prod + (YN(4) * (YO(35) * RCS(112))); \
    loss = loss + (YN(5) * RCS(113)); \
    prod = prod + (YN(1) * (YO(32) * RCS(114))); \
    loss = loss + (YN(6) * RCS(115)); \
    prod = prod + (YN(3) * (YO(32) * RCS(116))); \
    loss = loss + (YN(4) * RCS(117)); \
    prod = prod + (YN(6) * (YO(32) * RCS(122))); \
    loss = loss + ((YN(4) * YN(4)) * RCS(123)); \
    prod = prod + (YN(4) * (YO(32) * RCS(124))); \
    loss = loss + (YN(5) * RCS(125)); \
    prod = prod + (YO(32) * RCS(126)); \
    loss = loss + (YN(2) * RCS(127)); \
    rhs1 = rho * Y0S(1) + dt * WM(31) * (prod + extra); \
    rhs2 = -(dt * WM(31) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(31) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(31) - fnew); \
    UC_UPDATE_TAIL(31); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 33); \
    prod = (YN(30) * (YN(4) * RCS(68))); \
    extra = 0.0; \
    loss = (YN(5) * RCS(69)); \
    prod = prod + (YN(30) * (YN(2) * RCS(74))); \
    loss = loss + (YN(0) * RCS(75)); \
    prod = prod + (YN(30) * (YN(3) * RCS(80))); \
    loss = loss + (YN(4) * RCS(81)); \
    prod = prod + (YN(30) * (YN(13) * RCS(86))); \
    loss = loss + (YN(12) * RCS(87)); \
    prod = prod + (YN(30) * (YN(6) * RCS(90))); \
    loss = loss + (YN(7) * RCS(91)); \
    prod = prod + (YN(31) * (YN(6) * RCS(115))); \
    loss = loss + (YN(1) * RCS(114)); \
    prod = prod + (YN(31) * (YN(4) * RCS(117))); \
    loss = loss + (YN(3) * RCS(116)); \
    prod = prod + (YN(16) * (YN(5) * RCS(119))); \
    loss = loss + (YN(2) * RCS(118)); \
    prod = prod + (YN(28) * (YN(13) * RCS(121))); \
    loss = loss + (YN(2) * RCS(120)); \
    prod = prod + (YN(31) * ((YN(4) * YN(4)) * RCS(123))); \
    loss = loss + (YN(6) * RCS(122)); \
    prod = prod + (YN(31) * (YN(5) * RCS(125))); \
    loss = loss + (YN(4) * RCS(124)); \
    prod = prod + (YN(31) * (YN(2) * RCS(127))); \
    loss = loss + RCS(126); \
    rhs1 = rho * Y0S(0) + dt * WM(32) * (prod + extra); \
    rhs2 = -(dt * WM(32) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(32) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(32) - fnew); \
    UC_UPDATE_TAIL(32); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 34); \
    prod = (YN(30) * (YN(4) * RCS(66))); \
    extra = 0.0; \
    loss = (YN(5) * RCS(67)); \
    prod = prod + (YN(30) * (YN(2) * RCS(72))); \
    loss = loss + (YN(0) * RCS(73)); \
    prod = prod + (YN(30) * (YN(3) * RCS(78))); \
    loss = loss + (YN(4) * RCS(79)); \
    prod = prod + (YN(30) * (YN(13) * RCS(84))); \
    loss = loss + (YN(12) * RCS(85)); \
    prod = prod + (YN(30) * (YN(6) * RCS(92))); \
    loss = loss + (YN(7) * RCS(93)); \
    prod = prod + (YN(16) * (YN(4) * RCS(96))); \
    loss = loss + RCS(97); \
    rhs1 = rho * Y0S(1) + dt * WM(33) * (prod + extra); \
    rhs2 = -(dt * WM(33) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(33) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(33) - fnew); \
    UC_UPDATE_TAIL(33); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 35); \
    prod = (YN(13) * (YN(8) * RCS(39))); \
    extra = 0.0; \
    loss = RCS(38); \
    prod = prod + (YN(31) * (YN(4) * RCS(40))); \
    loss = loss + (YN(5) * RCS(41)); \
    prod = prod + (YN(31) * (YN(3) * RCS(44))); \
    loss = loss + (YN(4) * RCS(45)); \
    prod = prod + (YN(31) * (YN(2) * RCS(48))); \
    loss = loss + (YN(0) * RCS(49)); \
    prod = prod + (YN(31) * (YN(13) * RCS(52))); \
    loss = loss + (YN(12) * RCS(53)); \
    prod = prod + (YN(31) * (YN(6) * RCS(56))); \
    loss = loss + (YN(7) * RCS(57)); \
    prod = prod + (YN(31) * (YN(1) * RCS(60))); \
    loss = loss + (YN(6) * RCS(61)); \
    rhs1 = rho * Y0S(0) + dt * WM(34) * (prod + extra); \
    rhs2 = -(dt * WM(34) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(34) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(34) - fnew); \
    UC_UPDATE_TAIL(34); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 36); \
    prod = (YN(30) * (YN(4) * RCS(70))); \
    extra = 0.0; \
    loss = (YN(5) * RCS(71)); \
    prod = prod + (YN(30) * (YN(2) * RCS(76))); \
    loss = loss + (YN(0) * RCS(77)); \
    prod = prod + (YN(30) * (YN(3) * RCS(82))); \
    loss = loss + (YN(4) * RCS(83)); \
    prod = prod + (YN(30) * (YN(13) * RCS(88))); \
    loss = loss + (YN(12) * RCS(89)); \
    prod = prod + (YN(30) * (YN(6) * RCS(94))); \
    loss = loss + (YN(7) * RCS(95)); \
    prod = prod + (YN(18) * (YN(6) * RCS(98))); \
    loss = loss + (YN(4) * RCS(99)); \
    prod = prod + (YN(31) * (YN(2) * RCS(101))); \
    loss = loss + RCS(100); \
    prod = prod + (YN(13) * (YN(11) * RCS(103))); \
    loss = loss + RCS(102); \
    prod = prod + (YN(31) * (YN(6) * RCS(105))); \
    loss = loss + (YN(1) * RCS(104)); \
    prod = prod + (YN(18) * (YN(9) * RCS(107))); \
    loss = loss + (YN(8) * RCS(106)); \
    prod = prod + (YN(28) * (YN(13) * RCS(109))); \
    loss = loss + (YN(2) * RCS(108)); \
    prod = prod + (YN(16) * (YN(5) * RCS(111))); \
    loss = loss + (YN(2) * RCS(110)); \
    prod = prod + (YN(31) * (YN(5) * RCS(113))); \
    loss = loss + (YN(4) * RCS(112)); \
    rhs1 = rho * Y0S(1) + dt * WM(35) * (prod + extra); \
    rhs2 = -(dt * WM(35) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(35) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(35) - fnew); \
    UC_UPDATE_TAIL(35); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 37); \
    prod = (YN(16) * (YN(8) * RCS(129))); \
    extra = 0.0; \
    loss = (YN(3) * RCS(128)); \
    prod = prod + (YN(21) * (YN(13) * RCS(130))); \
    loss = loss + (YN(2) * RCS(131)); \
    prod = prod + (YN(26) * (YN(13) * RCS(133))); \
    loss = loss + (YN(3) * RCS(132)); \
    prod = prod + (YN(2) * (YO(37) * RCS(134))); \
    loss = loss + RCS(135); \
    prod = prod + (YN(6) * (YO(37) * RCS(136))); \
    loss = loss + (YN(1) * RCS(137)); \
    prod = prod + (YN(5) * (YO(37) * RCS(139))); \
    loss = loss + (YN(4) * RCS(138)); \
    prod = prod + (YO(38) * RCS(143)); \
    loss = loss + (YN(2) * RCS(142)); \
    prod = prod + (YN(2) * (YO(38) * RCS(144))); \
    loss = loss + (YN(0) * RCS(145)); \
    prod = prod + (YN(1) * (YO(38) * RCS(146))); \
    loss = loss + (YN(6) * RCS(147)); \
    prod = prod + (YN(13) * (YO(38) * RCS(148))); \
    loss = loss + (YN(12) * RCS(149)); \
    prod = prod + (YN(4) * (YO(38) * RCS(152))); \
    loss = loss + (YN(5) * RCS(153)); \
    prod = prod + (YN(10) * (YO(37) * RCS(154))); \
    loss = loss + (YN(8) * RCS(155)); \
    prod = prod + (YN(13) * ((YN(10) * YN(8)) * RCS(159))); \
    loss = loss + (YN(1) * RCS(158)); \
    prod = prod + (YO(45) * RCS(232)); \
    loss = loss + (YN(16) * RCS(233)); \
    prod = prod + (YN(1) * (YO(45) * RCS(238))); \
    loss = loss + ((YN(22) * YN(6)) * RCS(239)); \
    prod = prod + (YN(6) * (YO(45) * RCS(242))); \
    loss = loss + ((YN(22) * YN(7)) * RCS(243)); \
    rhs1 = rho * Y0S(0) + dt * WM(36) * (prod + extra); \
    rhs2 = -(dt * WM(36) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(36) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(36) - fnew); \
    UC_UPDATE_TAIL(36); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 38); \
    prod = (YN(36) * RCS(135)); \
    extra = 0.0; \
    loss = (YN(2) * RCS(134)); \
    prod = prod + (YN(36) * (YN(1) * RCS(137))); \
    loss = loss + (YN(6) * RCS(136)); \
    prod = prod + (YN(36) * (YN(4) * RCS(138))); \
    loss = loss + (YN(5) * RCS(139)); \
    prod = prod + (YN(25) * (YN(10) * RCS(141))); \
    loss = loss + (YN(1) * RCS(140)); \
    prod = prod + (YN(36) * (YN(8) * RCS(155))); \
    loss = loss + (YN(10) * RCS(154)); \
    prod = prod + (YN(22) * ((YN(4) * YN(8)) * RCS(157))); \
    loss = loss + (YN(6) * RCS(156)); \
    prod = prod + (YO(43) * RCS(229)); \
    loss = loss + (YN(13) * RCS(228)); \
    rhs1 = rho * Y0S(1) + dt * WM(37) * (prod + extra); \
    rhs2 = -(dt * WM(37) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(37) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(37) - fnew); \
    UC_UPDATE_TAIL(37); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 39); \
    prod = (YN(36) * (YN(2) * RCS(142))); \
    extra = 0.0; \
    loss = RCS(143); \
    prod = prod + (YN(36) * (YN(0) * RCS(145))); \
    loss = loss + (YN(2) * RCS(144)); \
    prod = prod + (YN(36) * (YN(6) * RCS(147))); \
    loss = loss + (YN(1) * RCS(146)); \
    prod = prod + (YN(36) * (YN(12) * RCS(149))); \
    loss = loss + (YN(13) * RCS(148)); \
    prod = prod + (YN(21) * (YN(13) * RCS(150))); \
    loss = loss + RCS(151); \
    prod = prod + (YN(36) * (YN(5) * RCS(153))); \
    loss = loss + (YN(4) * RCS(152)); \
    prod = prod + (YN(4) * (YO(39) * RCS(162))); \
    loss = loss + (YN(5) * RCS(163)); \
    prod = prod + (YN(2) * (YO(39) * RCS(166))); \
    loss = loss + (YN(0) * RCS(167)); \
    prod = prod + (YO(39) * RCS(169)); \
    loss = loss + (YN(2) * RCS(168)); \
    prod = prod + (YN(1) * (YO(39) * RCS(171))); \
    loss = loss + (YN(6) * RCS(170)); \
    prod = prod + (YN(22) * ((YN(4) * YN(11)) * RCS(173))); \
    loss = loss + (YN(6) * RCS(172)); \
    prod = prod + (YN(22) * (YN(13) * RCS(178))); \
    loss = loss + (YN(2) * RCS(179)); \
    prod = prod + (YN(4) * (YO(43) * RCS(224))); \
    loss = loss + ((YO(44) * YN(2)) * RCS(225)); \
    prod = prod + (YO(45) * RCS(234)); \
    loss = loss + (YN(22) * RCS(235)); \
    prod = prod + (YN(1) * (YO(45) * RCS(236))); \
    loss = loss + ((YN(21) * YN(6)) * RCS(237)); \
    prod = prod + (YN(6) * (YO(45) * RCS(240))); \
    loss = loss + ((YN(21) * YN(7)) * RCS(241)); \
    prod = prod + (YO(48) * RCS(262)); \
    loss = loss + (YN(18) * RCS(263)); \
    prod = prod + (YN(2) * (YO(48) * RCS(274))); \
    loss = loss + ((YN(0) * YN(16)) * RCS(275)); \
    prod = prod + (YO(47) * RCS(278)); \
    loss = loss + (YN(13) * RCS(279)); \
    rhs1 = rho * Y0S(0) + dt * WM(38) * (prod + extra); \
    rhs2 = -(dt * WM(38) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(38) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(38) - fnew); \
    UC_UPDATE_TAIL(38); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 40); \
    prod = (YN(18) * (YN(10) * RCS(161))); \
    extra = (1.0 * (YN(2) * (YO(46) * RCS(246)))); \
    loss = (YN(3) * RCS(160)); \
    prod = prod + (YN(38) * (YN(5) * RCS(163))); \
    extra = extra + (1.0 * (YN(4) * (YO(46) * RCS(258)))); \
    loss = loss + (YN(4) * RCS(162)); \
    prod = prod + (YN(25) * ((YN(13) * YN(2)) * RCS(165))); \
    loss = loss + (YN(3) * RCS(164)); \
    prod = prod + (YN(38) * (YN(0) * RCS(167))); \
    loss = loss + (YN(2) * RCS(166)); \
    prod = prod + (YN(38) * (YN(2) * RCS(168))); \
    loss = loss + RCS(169); \
    prod = prod + (YN(38) * (YN(6) * RCS(170))); \
    loss = loss + (YN(1) * RCS(171)); \
    prod = prod + (YN(22) * (YN(13) * RCS(174))); \
    loss = loss + RCS(175); \
    prod = prod + (YN(16) * (YN(13) * RCS(177))); \
    loss = loss + (YN(2) * RCS(176)); \
    prod = prod + (YO(41) * RCS(205)); \
    loss = loss + (YN(2) * RCS(204)); \
    prod = prod + (YN(1) * (YO(41) * RCS(206))); \
    loss = loss + (YN(6) * RCS(207)); \
    prod = prod + (YO(42) * RCS(211)); \
    loss = loss + (YN(2) * RCS(210)); \
    prod = prod + (YN(1) * (YO(42) * RCS(212))); \
    loss = loss + (YN(6) * RCS(213)); \
    prod = prod + (YO(45) * RCS(230)); \
    loss = loss + (YN(21) * RCS(231)); \
    prod = prod + (YO(48) * RCS(264)); \
    loss = loss + (YN(16) * RCS(265)); \
    prod = prod + (YN(4) * (YO(48) * RCS(266))); \
    loss = loss + ((YN(5) * YN(22)) * RCS(267)); \
    prod = prod + (YN(2) * (YO(48) * RCS(268))); \
    loss = loss + ((YN(0) * YN(22)) * RCS(269)); \
    prod = prod + (YN(2) * (YO(48) * RCS(272))); \
    loss = loss + (YN(18) * RCS(273)); \
    prod = prod + (YN(2) * (YO(47) * RCS(282))); \
    loss = loss + (YN(13) * RCS(283)); \
    rhs1 = rho * Y0S(1) + dt * WM(39) * (prod + extra); \
    rhs2 = -(dt * WM(39) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(39) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(39) - fnew); \
    UC_UPDATE_TAIL(39); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 41); \
    prod = (YN(18) * (YN(13) * RCS(181))); \
    extra = 0.0; \
    loss = RCS(180); \
    prod = prod + (YN(6) * (YO(41) * RCS(183))); \
    loss = loss + (YN(1) * RCS(182)); \
    prod = prod + (YN(6) * (YO(42) * RCS(185))); \
    loss = loss + (YN(1) * RCS(184)); \
    prod = prod + (YN(0) * (YO(41) * RCS(187))); \
    loss = loss + (YN(2) * RCS(186)); \
    prod = prod + (YN(0) * (YO(42) * RCS(189))); \
    loss = loss + (YN(2) * RCS(188)); \
    prod = prod + (YN(4) * (YO(41) * RCS(191))); \
    loss = loss + (YN(3) * RCS(190)); \
    prod = prod + (YN(4) * (YO(42) * RCS(193))); \
    loss = loss + (YN(3) * RCS(192)); \
    prod = prod + (YN(5) * (YO(42) * RCS(195))); \
    loss = loss + (YN(4) * RCS(194)); \
    prod = prod + (YN(5) * (YO(41) * RCS(197))); \
    loss = loss + (YN(4) * RCS(196)); \
    prod = prod + (YN(7) * (YO(41) * RCS(199))); \
    loss = loss + (YN(6) * RCS(198)); \
    prod = prod + (YN(7) * (YO(42) * RCS(201))); \
    loss = loss + (YN(6) * RCS(200)); \
    rhs1 = rho * Y0S(0) + dt * WM(40) * (prod + extra); \
    rhs2 = -(dt * WM(40) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(40) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(40) - fnew); \
    UC_UPDATE_TAIL(40); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 42); \
    prod = (YN(40) * (YN(1) * RCS(182))); \
    extra = 0.0; \
    loss = (YN(6) * RCS(183)); \
    prod = prod + (YN(40) * (YN(2) * RCS(186))); \
    loss = loss + (YN(0) * RCS(187)); \
    prod = prod + (YN(40) * (YN(3) * RCS(190))); \
    loss = loss + (YN(4) * RCS(191)); \
    prod = prod + (YN(40) * (YN(4) * RCS(196))); \
    loss = loss + (YN(5) * RCS(197)); \
    prod = prod + (YN(40) * (YN(6) * RCS(198))); \
    loss = loss + (YN(7) * RCS(199)); \
    prod = prod + (YO(42) * RCS(203)); \
    loss = loss + RCS(202); \
    prod = prod + (YN(39) * (YN(2) * RCS(204))); \
    loss = loss + RCS(205); \
    prod = prod + (YN(39) * (YN(6) * RCS(207))); \
    loss = loss + (YN(1) * RCS(206)); \
    rhs1 = rho * Y0S(1) + dt * WM(41) * (prod + extra); \
    rhs2 = -(dt * WM(41) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(41) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(41) - fnew); \
    UC_UPDATE_TAIL(41); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 43); \
    prod = (YN(40) * (YN(1) * RCS(184))); \
    extra = 0.0; \
    loss = (YN(6) * RCS(185)); \
    prod = prod + (YN(40) * (YN(2) * RCS(188))); \
    loss = loss + (YN(0) * RCS(189)); \
    prod = prod + (YN(40) * (YN(3) * RCS(192))); \
    loss = loss + (YN(4) * RCS(193)); \
    prod = prod + (YN(40) * (YN(4) * RCS(194))); \
    loss = loss + (YN(5) * RCS(195)); \
    prod = prod + (YN(40) * (YN(6) * RCS(200))); \
    loss = loss + (YN(7) * RCS(201)); \
    prod = prod + (YN(41) * RCS(202)); \
    loss = loss + RCS(203); \
    prod = prod + (YN(16) * (YN(13) * RCS(209))); \
    loss = loss + RCS(208); \
    prod = prod + (YN(39) * (YN(2) * RCS(210))); \
    loss = loss + RCS(211); \
    prod = prod + (YN(39) * (YN(6) * RCS(213))); \
    loss = loss + (YN(1) * RCS(212)); \
    rhs1 = rho * Y0S(0) + dt * WM(42) * (prod + extra); \
    rhs2 = -(dt * WM(42) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(42) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(42) - fnew); \
    UC_UPDATE_TAIL(42); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 44); \
    prod = (YN(22) * ((YN(21) * YN(2)) * RCS(215))); \
    extra = 0.0; \
    loss = RCS(214); \
    prod = prod + (YN(22) * (YOS(7) * RCS(217))); \
    loss = loss + RCS(216); \
    prod = prod + (YN(22) * (YOS(7) * RCS(218))); \
    loss = loss + RCS(219); \
    prod = prod + (YN(22) * (YN(16) * RCS(221))); \
    loss = loss + (YN(2) * RCS(220)); \
    prod = prod + (YN(22) * ((YN(0) * YN(21)) * RCS(223))); \
    loss = loss + (YN(2) * RCS(222)); \
    prod = prod + (YN(38) * ((YO(44) * YN(2)) * RCS(225))); \
    loss = loss + (YN(4) * RCS(224)); \
    prod = prod + (YN(22) * ((YN(12) * YN(21)) * RCS(227))); \
    loss = loss + (YN(13) * RCS(226)); \
    prod = prod + (YN(37) * (YN(13) * RCS(228))); \
    loss = loss + RCS(229); \
    prod = prod + (YN(2) * (YO(48) * RCS(276))); \
    loss = loss + ((YN(0) * YN(13)) * RCS(277)); \
    prod = prod + (YN(4) * (YO(47) * RCS(286))); \
    loss = loss + ((YN(5) * YN(2)) * RCS(287)); \
    rhs1 = rho * Y0S(1) + dt * WM(43) * (prod + extra); \
    rhs2 = -(dt * WM(43) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(43) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(43) - fnew); \
    UC_UPDATE_TAIL(43); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 45); \
    prod = (YN(43) * (YN(4) * RCS(224))); \
    extra = 0.0; \
    loss = ((YN(2) * YN(38)) * RCS(225)); \
    rhs1 = rho * Y0S(0) + dt * WM(44) * (prod + extra); \
    rhs2 = -(dt * WM(44) * loss); \
    ppp = rho - FSS(0); \
    fnew = sor2 * YO(44) + (rhs1 - FNS(0)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(44) - fnew); \
    UC_UPDATE_TAIL(44); \
    UC_TR_SYNC(); \
    UC_TR_PF(0, 46); \
    prod = (YN(39) * (YN(21) * RCS(231))); \
    extra = 0.0; \
    loss = RCS(230); \
    prod = prod + (YN(36) * (YN(16) * RCS(233))); \
    loss = loss + RCS(232); \
    prod = prod + (YN(38) * (YN(22) * RCS(235))); \
    loss = loss + RCS(234); \
    prod = prod + (YN(38) * ((YN(21) * YN(6)) * RCS(237))); \
    loss = loss + (YN(1) * RCS(236)); \
    prod = prod + (YN(36) * ((YN(22) * YN(6)) * RCS(239))); \
    loss = loss + (YN(1) * RCS(238)); \
    prod = prod + (YN(38) * ((YN(21) * YN(7)) * RCS(241))); \
    loss = loss + (YN(6) * RCS(240)); \
    prod = prod + (YN(36) * ((YN(22) * YN(7)) * RCS(243))); \
    loss = loss + (YN(6) * RCS(242)); \
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
    loss = RCS(244); \
    prod = prod + 0.0; \
    loss = loss + (YN(2) * RCS(246)); \
    prod = prod + 0.0; \
    loss = loss + (YN(2) * RCS(248)); \
    prod = prod + 0.0; \
    loss = loss + (YN(2) * RCS(250)); \
    prod = prod + (YN(18) * ((YN(0) * YO(48)) * RCS(253))); \
    loss = loss + (YN(2) * RCS(252)); \
    prod = prod + (YN(18) * ((YN(5) * YO(48)) * RCS(255))); \
    loss = loss + (YN(4) * RCS(254)); \
    prod = prod + 0.0; \
    loss = loss + (YN(4) * RCS(256)); \
    prod = prod + 0.0; \
    loss = loss + (YN(4) * RCS(258)); \
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
    prod = (YN(38) * (YN(13) * RCS(279))); \
    extra = (1.0 * (YN(46) * (YN(2) * RCS(248)))); \
    loss = RCS(278); \
    prod = prod + (YN(18) * (YN(16) * RCS(281))); \
    extra = extra + (1.0 * (YN(46) * (YN(4) * RCS(256)))); \
    loss = loss + (YN(2) * RCS(280)); \
    prod = prod + (YN(39) * (YN(13) * RCS(283))); \
    loss = loss + (YN(2) * RCS(282)); \
    prod = prod + (YN(22) * ((YN(0) * YN(16)) * RCS(285))); \
    loss = loss + (YN(2) * RCS(284)); \
    prod = prod + (YN(43) * ((YN(5) * YN(2)) * RCS(287))); \
    loss = loss + (YN(4) * RCS(286)); \
    rhs1 = rho * Y0S(1) + dt * WM(47) * (prod + extra); \
    rhs2 = -(dt * WM(47) * loss); \
    ppp = rho - FSS(1); \
    fnew = sor2 * YO(47) + (rhs1 - FNS(1)) * sor1 / (ppp - rhs2); \
    rsd += fabs(YO(47) - fnew); \
    UC_UPDATE_TAIL(47); \
    UC_TR_SYNC(); \
    UC_TR_PF(1, 49); \
    prod = (YN(46) * (YN(2) * RCS(252))); \
    extra = 0.0; \
    loss = ((YN(0) * YN(18)) * RCS(253)); \
    prod = prod + (YN(46) * (YN(4) * RCS(254))); \
    loss = loss + ((YN(5) * YN(18)) * RCS(255)); \
    prod = prod + (YN(38) * (YN(18) * RCS(263))); \
    loss = loss + RCS(262); \
    prod = prod + (YN(39) * (YN(16) * RCS(265))); \
    loss = loss + RCS(264); \
    prod = prod + (YN(39) * ((YN(5) * YN(22)) * RCS(267))); \
    loss = loss + (YN(4) * RCS(266)); \
    prod = prod + (YN(39) * ((YN(0) * YN(22)) * RCS(269))); \
    loss = loss + (YN(2) * RCS(268)); \
    prod = prod + (YN(16) * ((YOS(4) * YN(13)) * RCS(271))); \
    loss = loss + (YN(2) * RCS(270)); \
    prod = prod + (YN(39) * (YN(18) * RCS(273))); \
    loss = loss + (YN(2) * RCS(272)); \
    prod = prod + (YN(38) * ((YN(0) * YN(16)) * RCS(275))); \
    loss = loss + (YN(2) * RCS(274)); \
    prod = prod + (YN(43) * ((YN(0) * YN(13)) * RCS(277))); \
    loss = loss + (YN(2) * RCS(276)); \
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
static __constant__ int16_t uc_tr_trow[256] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51, 52, 53, 54, 55, 56, 57, 58, 59, 60, 61, 62, 63, 64, 65, 66, 67, 68, 69, 70, 71, 72, 73, 74, 75, 76, 77, 78, 79, 80, 81, 82, 83, 84, 85, 86, 87, 88, 89, 90, 91, 92, 93, 94, 95, 96, 97, 98, 99, 100, 101, 102, 103, 104, 105, 106, 107, 108, 109, 110, 111, 112, 113, 114, 115, 116, 117, 118, 119, 120, 121, 122, 123, 124, 125, 126, 127, 128, 129, 130, 131, 132, 133, 134, 135, 136, 137, 138, 139, 140, 141, 142, 143, 144, 145, 146, 147, 148, 149, 150, 151, 152, 153, 154, 155, 156, 157, 158, 159, 160, 161, 162, 163, 164, 165, 166, 167, 168, 169, 170, 171, 172, 173, 174, 175, 176, 177, 178, 179, 180, 181, 182, 183, 184, 185, 186, 187, 188, 189, 190, 191, 192, 193, 194, 195, 196, 197, 198, 199, 200, 201, 202, 203, 204, 205, 206, 207, 208, 209, 210, 211, 212, 213, 214, 215, 216, 217, 218, 219, 220, 221, 222, 223, 224, 225, 226, 227, 228, 229, 230, 231, 232, 233, 234, 235, 236, 237, 238, 239, 240, 241, 242, 243, 244, 245, 246, 247, 248, 249, 250, 251, 252, 253, 254, 255};
static __constant__ int16_t uc_tr_srow[288] = {256, 257, 258, 259, 260, 261, 262, 263, 264, 265, 266, 267, 268, 269, 270, 271, 272, 273, 274, 275, 276, 277, 278, 279, 280, 281, 282, 283, 284, 285, 286, 287, 288, 289, 290, 291, 292, 293, 294, 295, 296, 297, 298, 299, 300, 301, 302, 303, 304, 305, 306, 307, 308, 309, 310, 311, 312, 313, 314, 315, 316, 317, 318, 319, 320, 321, 322, 323, 324, 325, 326, 327, 328, 329, 330, 331, 332, 333, 334, 335, 336, 337, 338, 339, 340, 341, 342, 343, 344, 345, 346, 347, 348, 349, 350, 351, 352, 353, 354, 355, 356, 357, 358, 359, 360, 361, 362, 363, 364, 365, 366, 367, 368, 369, 370, 371, 372, 373, 374, 375, 376, 377, 378, 379, 380, 381, 382, 383, 384, 385, 386, 387, 388, 389, 390, 391, 392, 393, 394, 395, 396, 397, 398, 399, 400, 401, 402, 403, 404, 405, 406, 407, 408, 409, 410, 411, 412, 413, 414, 415, 416, 417, 418, 419, 420, 421, 422, 423, 424, 425, 426, 427, 428, 429, 430, 431, 432, 433, 434, 435, 436, 437, 438, 439, 440, 441, 442, 443, 444, 445, 446, 447, 448, 449, 450, 451, 452, 453, 454, 455, 456, 457, 458, 459, 460, 461, 462, 463, 464, 465, 466, 467, 468, 469, 470, 471, 472, 473, 474, 475, 476, 477, 478, 479, 480, 481, 482, 483, 484, 485, 486, 487, 488, 489, 490, 491, 492, 493, 494, 495, 496, 497, 498, 499, 500, 501, 502, 503, 504, 505, 506, 507, 508, 509, 510, 511, 512, 513, 514, 515, 516, 517, 518, 519, 520, 521, 522, 523, 524, 525, 526, 527, 528, 529, 530, 531, 532, 533, 534, 535, 536, 537, 538, 539, 540, 541, 542, 543};
#else
static const short uc_tr_trow[256] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51, 52, 53, 54, 55, 56, 57, 58, 59, 60, 61, 62, 63, 64, 65, 66, 67, 68, 69, 70, 71, 72, 73, 74, 75, 76, 77, 78, 79, 80, 81, 82, 83, 84, 85, 86, 87, 88, 89, 90, 91, 92, 93, 94, 95, 96, 97, 98, 99, 100, 101, 102, 103, 104, 105, 106, 107, 108, 109, 110, 111, 112, 113, 114, 115, 116, 117, 118, 119, 120, 121, 122, 123, 124, 125, 126, 127, 128, 129, 130, 131, 132, 133, 134, 135, 136, 137, 138, 139, 140, 141, 142, 143, 144, 145, 146, 147, 148, 149, 150, 151, 152, 153, 154, 155, 156, 157, 158, 159, 160, 161, 162, 163, 164, 165, 166, 167, 168, 169, 170, 171, 172, 173, 174, 175, 176, 177, 178, 179, 180, 181, 182, 183, 184, 185, 186, 187, 188, 189, 190, 191, 192, 193, 194, 195, 196, 197, 198, 199, 200, 201, 202, 203, 204, 205, 206, 207, 208, 209, 210, 211, 212, 213, 214, 215, 216, 217, 218, 219, 220, 221, 222, 223, 224, 225, 226, 227, 228, 229, 230, 231, 232, 233, 234, 235, 236, 237, 238, 239, 240, 241, 242, 243, 244, 245, 246, 247, 248, 249, 250, 251, 252, 253, 254, 255};
static const short uc_tr_srow[288] = {256, 257, 258, 259, 260, 261, 262, 263, 264, 265, 266, 267, 268, 269, 270, 271, 272, 273, 274, 275, 276, 277, 278, 279, 280, 281, 282, 283, 284, 285, 286, 287, 288, 289, 290, 291, 292, 293, 294, 295, 296, 297, 298, 299, 300, 301, 302, 303, 304, 305, 306, 307, 308, 309, 310, 311, 312, 313, 314, 315, 316, 317, 318, 319, 320, 321, 322, 323, 324, 325, 326, 327, 328, 329, 330, 331, 332, 333, 334, 335, 336, 337, 338, 339, 340, 341, 342, 343, 344, 345, 346, 347, 348, 349, 350, 351, 352, 353, 354, 355, 356, 357, 358, 359, 360, 361, 362, 363, 364, 365, 366, 367, 368, 369, 370, 371, 372, 373, 374, 375, 376, 377, 378, 379, 380, 381, 382, 383, 384, 385, 386, 387, 388, 389, 390, 391, 392, 393, 394, 395, 396, 397, 398, 399, 400, 401, 402, 403, 404, 405, 406, 407, 408, 409, 410, 411, 412, 413, 414, 415, 416, 417, 418, 419, 420, 421, 422, 423, 424, 425, 426, 427, 428, 429, 430, 431, 432, 433, 434, 435, 436, 437, 438, 439, 440, 441, 442, 443, 444, 445, 446, 447, 448, 449, 450, 451, 452, 453, 454, 455, 456, 457, 458, 459, 460, 461, 462, 463, 464, 465, 466, 467, 468, 469, 470, 471, 472, 473, 474, 475, 476, 477, 478, 479, 480, 481, 482, 483, 484, 485, 486, 487, 488, 489, 490, 491, 492, 493, 494, 495, 496, 497, 498, 499, 500, 501, 502, 503, 504, 505, 506, 507, 508, 509, 510, 511, 512, 513, 514, 515, 516, 517, 518, 519, 520, 521, 522, 523, 524, 525, 526, 527, 528, 529, 530, 531, 532, 533, 534, 535, 536, 537, 538, 539, 540, 541, 542, 543};
#endif
