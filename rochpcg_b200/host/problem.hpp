// The C ABI problem handle: one HPCG hierarchy with its CG vectors.
#pragma once

#include <vector>

#include "hpcg.hpp"

struct hpcgb200_problem
{
    Geometry* geom = nullptr;
    SparseMatrix A{};
    Vector b, x, xexact;
    CGData data{};
    int nlevels = 0;
    double setup_s = 0.0, optimize_s = 0.0;
    double* b_generated = nullptr;  // permuted generated b (restored by set_rhs(NULL))
    std::vector<SparseMatrix*> levels;
};
