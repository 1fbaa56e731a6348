// Polygon triangulations used by edge swapping (edge_swap.cpp:21-228).
//
// For a ring of N vertices (3..7) every triangulation of the N-gon is listed
// in a fixed order; the order decides which triangulation wins a quality tie
// (choose_edge_swap, edge_swap.cpp:230-280) and the order of the entities a
// swap emits (get_swap_ents, edge_swap.cpp:282-373), so it must match the
// reference exactly. Each triangulation lists its N-2 triangles as three
// ring-vertex digits; triangulations are separated by spaces, triangles by
// dots. The interior edges of each triangulation are derived from these
// triangles at start-up (edge_swap.cu).
#pragma once

namespace osh {

static char const* const polygon_triangulations[8] = {
  nullptr, nullptr, nullptr,
  /* 3 */ "012",
  /* 4 */ "012.023 013.123",
  /* 5 */ "012.023.034 014.134.123 012.234.024 034.123.013 014.234.124",
  /* 6 */ "012.023.034.045 012.025.245.234 012.023.035.345 012.045.234.024 "
          "012.025.345.235 034.045.123.013 123.015.145.134 035.345.123.013 "
          "045.123.134.014 345.123.015.135 234.015.145.124 045.234.014.124 "
          "245.234.015.125 345.235.015.125",
  /* 7 */ "012.023.034.045.056 012.023.036.356.345 012.023.034.046.456 "
          "012.023.056.345.035 012.023.036.456.346 012.045.056.024.234 "
          "012.234.026.256.245 012.046.456.024.234 012.056.234.245.025 "
          "012.456.234.026.246 012.345.026.256.235 012.056.345.025.235 "
          "012.356.345.026.236 012.456.346.026.236 034.045.056.013.123 "
          "036.356.345.013.123 034.046.456.013.123 056.345.035.013.123 "
          "036.456.346.013.123 045.056.123.014.134 123.134.016.156.145 "
          "046.456.123.014.134 056.123.134.145.015 456.123.134.016.146 "
          "345.123.016.156.135 056.345.123.015.135 356.345.123.016.136 "
          "456.346.123.016.136 045.056.234.014.124 234.016.156.145.124 "
          "046.456.234.014.124 056.234.145.015.124 456.234.016.146.124 "
          "234.245.016.156.125 056.234.245.015.125 234.256.245.016.126 "
          "456.234.246.016.126 345.235.016.156.125 056.345.235.015.125 "
          "345.256.235.016.126 356.345.236.016.126 456.346.236.016.126"
};

}  // namespace osh
