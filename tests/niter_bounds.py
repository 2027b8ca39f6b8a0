"""The reference's pinned CG iteration bounds (src/test_rochpcg.cpp:88-119,
`check_niter`): the optimized CG, run to the tolerance 50 CG_ref iterations
reach, must stop within these many iterations for a rank count and a cubic
local brick; every other case is held to 50."""

_BOUNDS = {
    (1, 16): 53, (2, 16): 53, (4, 16): 56, (1, 32): 53, (4, 32): 55, (2, 48): 52, (4, 48): 55,
    (2, 64): 52, (4, 64): 52, (2, 80): 53, (4, 80): 54, (2, 96): 52, (4, 96): 51, (1, 104): 53,
    (2, 104): 51, (4, 104): 51, (2, 112): 51, (4, 112): 51, (2, 120): 51, (4, 120): 51, (2, 128): 51,
    (4, 128): 51, (1, 256): 52, (2, 256): 52, (4, 256): 52, (1, 288): 51, (2, 288): 51, (4, 288): 51,
}


def check_niter(size: int, dims) -> int:
    nx, ny, nz = dims
    if nx == ny == nz:
        return _BOUNDS.get((size, nx), 50)
    return 50
