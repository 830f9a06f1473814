// Force-included when the reference's kernel sources are compiled as host C++.
//
// Test infrastructure only: this builds the CHECKER (oracle/_ref), never the product.
//
// The reference declares `template <typename T> struct Distance;` only under UNITTEST
// (kernel/ocl/algebra/real.hh:59-65) but specialises it under HOST
// (e.g. kernel/ocl/transform/shift.hh:16-23, kernel/ocl/transform/moebius.hh:28-35),
// so a HOST-only build needs the primary template declared up front.
#pragma once
#include <types.hh>
template <typename T> struct Distance;
