/*
 * Stand-in for <boost/random.hpp> used only to compile the reference's
 * headers into the CPU oracle.  The reference names boost::random::mt19937
 * and uniform_real_distribution<double> in include/Math/random.h:58-60; the
 * flow path never draws from them (Metropolis only), so the standard-library
 * engines with the same interface are enough.  Test infrastructure.
 */
#pragma once
#include <random>
namespace boost { namespace random {
using mt19937 = std::mt19937;
template <class T> using uniform_real_distribution = std::uniform_real_distribution<T>;
} }
