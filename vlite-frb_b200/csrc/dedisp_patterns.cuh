// Generated by gen_patterns.py -- do not edit.
// In-group delay patterns (0, Delta_1, ..., Delta_{D-1}) of D adjacent,
// equally spaced DM trials: Delta_j = floor(phi + j*y) (see gen_patterns.py).
#pragma once

#define VFRB_PAT4_SMAX 20
#define VFRB_PAT4_N 49
// X(id, Delta_1, ..., Delta_3)
#define VFRB_PAT4_LIST(X) \
  X(0, 0, 0, 0) X(1, 0, 0, 1) X(2, 0, 1, 1) X(3, 1, 1, 1) X(4, 0, 1, 2) X(5, 1, 1, 2) \
  X(6, 1, 2, 2) X(7, 1, 2, 3) X(8, 1, 2, 4) X(9, 1, 3, 4) X(10, 2, 3, 4) X(11, 1, 3, 5) \
  X(12, 2, 3, 5) X(13, 2, 4, 5) X(14, 2, 4, 6) X(15, 2, 4, 7) X(16, 2, 5, 7) X(17, 3, 5, 7) \
  X(18, 2, 5, 8) X(19, 3, 5, 8) X(20, 3, 6, 8) X(21, 3, 6, 9) X(22, 3, 6, 10) X(23, 3, 7, 10) \
  X(24, 4, 7, 10) X(25, 3, 7, 11) X(26, 4, 7, 11) X(27, 4, 8, 11) X(28, 4, 8, 12) X(29, 4, 8, 13) \
  X(30, 4, 9, 13) X(31, 5, 9, 13) X(32, 4, 9, 14) X(33, 5, 9, 14) X(34, 5, 10, 14) X(35, 5, 10, 15) \
  X(36, 5, 10, 16) X(37, 5, 11, 16) X(38, 6, 11, 16) X(39, 5, 11, 17) X(40, 6, 11, 17) X(41, 6, 12, 17) \
  X(42, 6, 12, 18) X(43, 6, 12, 19) X(44, 6, 13, 19) X(45, 7, 13, 19) X(46, 6, 13, 20) X(47, 7, 13, 20) \
  X(48, 7, 14, 20)

#define VFRB_PAT2_SMAX 16
#define VFRB_PAT2_N 17
// X(id, Delta_1, ..., Delta_1)
#define VFRB_PAT2_LIST(X) \
  X(0, 0) X(1, 1) X(2, 2) X(3, 3) X(4, 4) X(5, 5) \
  X(6, 6) X(7, 7) X(8, 8) X(9, 9) X(10, 10) X(11, 11) \
  X(12, 12) X(13, 13) X(14, 14) X(15, 15) X(16, 16)
