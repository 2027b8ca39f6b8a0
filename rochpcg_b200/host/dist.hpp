// Domain decomposition of the HPCG problem over ranks (one GPU each): process
// grid, per-level halo plan and the distributed problem handle.
//
// Reference behaviour restated here:
//  * process grid: src/ComputeOptimalShapeXYZ.cpp:94-157 (prime factors of the
//    rank count dealt into three dimensions of least surface), rank
//    coordinates src/GenerateGeometry.cpp:84-86, global offsets :126-166;
//  * halo plan: src/SetupHalo.cpp:135-292,294-651 -- neighbours numbered by
//    their relative position (dz,dy,dx) in [-1,1]^3, slot 13 being the rank
//    itself; the external columns received from a neighbour are its global
//    ids in ascending order, numbered after the local rows neighbour by
//    neighbour in slot order; the rows sent to a neighbour are the local rows
//    with a column in its domain, ascending;
//  * optimized matrix: the local ELL keeps the single-rank column order for
//    the local columns (src/Permute.cpp:95-185 sorts keys perm[col] for local
//    columns, the external id for external ones, so external columns follow
//    the local ones in ascending external id), and the rows with external
//    columns are listed in ascending natural order with their external
//    entries (src/SparseMatrix.cpp:166-269, kernel_to_ell_col/kernel_to_halo).
#pragma once

#include <vector>

namespace hpcg_b200 {

// src/ComputeOptimalShapeXYZ.cpp:94-157 (the default, non-cubic-radical search).
void optimal_shape(int size, int& npx, int& npy, int& npz);

struct DistGeom
{
    int size = 1, rank = 0;
    int npx = 1, npy = 1, npz = 1;
    int ipx = 0, ipy = 0, ipz = 0;
    int nx = 0, ny = 0, nz = 0;          // local brick of this level
    long long gnx = 0, gny = 0, gnz = 0; // global grid of this level
    long long gix0 = 0, giy0 = 0, giz0 = 0;

    // the rank at process-grid coordinates (px, py, pz)
    int rank_at(int px, int py, int pz) const { return px + py * npx + pz * npx * npy; }
};

// src/GenerateGeometry.cpp:84-86,126-166 (one z partition: every rank has the
// same local brick).  npx*npy*npz == size is required.
DistGeom make_geom(int size, int rank, int npx, int npy, int npz, int nx, int ny, int nz);
// The next coarser level's geometry: every local extent halved.
DistGeom coarsen(const DistGeom& g);

struct HaloPlan
{
    int m = 0;                           // local rows
    int next = 0;                        // external columns (ids m .. m+next-1)
    std::vector<int> nbr_rank;           // neighbours in slot order
    std::vector<int> nbr_slot;           // their slots (dz+1)*9 + (dy+1)*3 + (dx+1)
    std::vector<int> recv_len, recv_off; // external ids received from each neighbour: [m+off, m+off+len)
    std::vector<int> send_len, send_off; // rows sent to each neighbour: send_rows[off, off+len)
    std::vector<long long> recv_gid;     // global id of external column m+e
    std::vector<int> send_rows;          // natural local rows, ascending per neighbour
    std::vector<int> halo_rows;          // natural rows with external columns, ascending
    std::vector<int> halo_ptr;           // halo row h owns halo_cols[halo_ptr[h], halo_ptr[h+1])
    std::vector<int> halo_cols;          // its external columns (m+e), ascending
    int halo_width = 0;                  // most external columns of one row
};

HaloPlan plan_halo(const DistGeom& g);

}  // namespace hpcg_b200
