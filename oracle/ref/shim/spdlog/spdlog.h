/* Minimal logging sink standing in for spdlog in the reference build (stderr). */
#pragma once
#include <cstdlib>
#include <iostream>
#include <string>
namespace spdlog {
inline bool quiet() { static const bool q = std::getenv("VTREF_VERBOSE") == nullptr; return q; }
template <class T> void info(const T &m) { if (!quiet()) std::cerr << "[info] " << m << "\n"; }
template <class T> void warn(const T &m) { if (!quiet()) std::cerr << "[warn] " << m << "\n"; }
template <class T> void error(const T &m) { std::cerr << "[error] " << m << "\n"; }
}  // namespace spdlog
