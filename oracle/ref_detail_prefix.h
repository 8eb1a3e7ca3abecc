/*
 * ref_detail_prefix.h -- TEST INFRASTRUCTURE (oracle), never part of the
 * product.
 *
 * The reference's detail-preserving tone map lives in the LibRaw-dependent
 * wrapper (core/libraw_wrapper.cpp) but uses nothing of LibRaw: the free
 * function box_filter_normalized (:45-116) and the member functions
 * aces_tone_map_scalar + apply_detail_preserving_tonemap (:1389-1471).
 * oracle/Makefile streams exactly those two line ranges from the reference
 * source, in this order:
 *
 *     ref_detail_prefix.h, lines 45-116, ref_detail_mid.h,
 *     lines 1389-1471, ref_detail_suffix.h
 *
 * into oracle/_ref/liblre_ref_dt.so.  Nothing of the reference is copied
 * into the repository.  GCC ignores the reference's clang-only
 * `#pragma float_control`; the recipe's -ffp-contract=off and no fast-math
 * give the precise semantics that pragma asks for.
 */
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <iostream>
#include <vector>

#include "accelerator.h"

namespace libraw_enhanced {
