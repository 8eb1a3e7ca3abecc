/*
 * ref_highlights_prefix.h -- TEST INFRASTRUCTURE (oracle), never part of the
 * product.
 *
 * The reference's highlight recovery is a member of the LibRaw-dependent
 * wrapper class (core/libraw_wrapper.cpp:1095-1383) but uses nothing of the
 * class or of LibRaw.  oracle/Makefile compiles exactly those lines, streamed
 * from the reference source, between this prefix and
 * ref_highlights_suffix.h, into oracle/_ref/liblre_ref_hl.so.  Nothing of the
 * reference is copied into the repository.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <iostream>
#include <limits>
#include <vector>

#include "accelerator.h"

namespace libraw_enhanced {
struct RefHighlights {
