// Enumeration of the unordered neighbour pairs of an angular group in rounds
// of matchings, shared by the Gaussian (sf_fast.cuh) and compact
// (k_compact.cu) symmetry-function kernels.
#pragma once

namespace n2p2b200 {

namespace {

// Candidate pairs of one angular group, each unordered pair once, enumerated
// in rounds of matchings (no slot occurs twice in one round, which lets the
// force pass add a round's contributions without conflicts):
//   kind 3  tournament over one block of nO slots (circle method on
//           m = nO rounded up to even): round r < m - 1 pairs (m - 1, r) and
//           ((r + i) mod (m - 1), (r - i) mod (m - 1)) for 0 < i < m / 2;
//           slot m - 1 = nO (odd nO) is a bye
//   kind 4  diagonals between blocks nO <= D: round r < D pairs owner a
//           with partner (a + r) mod D, a < nO
// The cursor walks the round a and the index t < minor within the round.
struct Phase
{
    int kind, O0, nO, P0, D, count, minor;
};

// Thread-private decoding of candidate p (init), advanced by 32 per step or
// by a fixed stride without integer division in the loop.
struct Cursor
{
    int a, t;
    __device__ __forceinline__ void init(Phase const& ph, int p)
    {
        a = p / ph.minor;
        t = p - a * ph.minor;
    }
    __device__ __forceinline__ void advance(Phase const& ph)
    {
        t += 32;
        while (t >= ph.minor)
        {
            t -= ph.minor;
            ++a;
        }
    }
    // Advance by a stride of q * minor + rem (rem < minor) candidates.
    __device__ __forceinline__ void advance(Phase const& ph, int q, int rem)
    {
        a += q;
        t += rem;
        if (t >= ph.minor)
        {
            t -= ph.minor;
            ++a;
        }
    }
    // Slots of the candidate; false for a bye.
    __device__ __forceinline__ bool slots(Phase const& ph, int& so, int& sp) const
    {
        if (ph.kind == 3)
        {
            const int m1 = ph.nO - 1 + (ph.nO & 1);
            int u, v;
            if (t == 0)
            {
                u = m1;
                v = a;
            }
            else
            {
                u = a + t;
                if (u >= m1) u -= m1;
                v = a - t;
                if (v < 0) v += m1;
            }
            so = ph.O0 + u;
            sp = ph.O0 + v;
            return u < ph.nO;
        }
        int q = t + a;
        if (q >= ph.D) q -= ph.D;
        so = ph.O0 + t;
        sp = ph.P0 + q;
        return true;
    }
    // Round of the candidate, 11 bits.
    __device__ __forceinline__ int round(Phase const&) const { return a & 0x7ff; }
};

// The unordered pairs of a group as rounds of matchings (both passes).
__device__ __forceinline__ int roundPhases(int A0, int nA, int B0, int nB, bool same, Phase* ph)
{
    if (same)
    {
        if (nA < 2) return 0;
        const int m = nA + (nA & 1);
        ph[0] = Phase{3, A0, nA, A0, 0, (m - 1) * (m / 2), m / 2};
        return 1;
    }
    if (nA == 0 || nB == 0) return 0;
    if (nA <= nB) ph[0] = Phase{4, A0, nA, B0, nB, nA * nB, nA};
    else ph[0] = Phase{4, B0, nB, A0, nA, nA * nB, nB};
    return 1;
}

} // namespace

} // namespace n2p2b200
