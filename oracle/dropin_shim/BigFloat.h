/* Drop-in check: stands in for the reference's BigFloat.h when the
 * reference's own PI.h is compiled UNMODIFIED against this library's C++
 * BigFloat (oracle/Makefile target `dropin`).  The reference's Pi() and
 * Pi_BSR() (PI.h:64-212) then run every product, add, reciprocal and inverse
 * square root on the GPU through pic::BigFloat, whose public API is the
 * reference's (BigFloat.h:10-30, 46). */
#pragma once
#include "bigfloat.hpp"
#include "piculator_b200.h"

using pic::BigFloat;
using pic::invsqrt;
