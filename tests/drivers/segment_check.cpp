// Host check of the bulk segments the builder makes: every lane of a segment
// has the neighbours the per-cell decode gives, no lane's +1 neighbours wrap
// (those cells must be listed), and every cell that is not solid is collided
// exactly once (one segment lane, the special list or the rotor list).
#include "../../lbm3_b200/csrc/builder.h"

#include <cstdio>
#include <vector>

extern "C" int lbm_segment_check(const lbm_case* c, long long* segments, long long* longest) {
    lbm::HostDomain d;
    lbm::buildDomain(*c, d);
    int bad = 0;
    *segments = 0;
    *longest = 0;
    for (const lbm::HostLevel& L : d.levels) {
        const int n = L.info.cellCount;
        std::vector<int> covered(n, 0);
        for (size_t s = 0; s < L.segCell.size(); ++s) {
            ++*segments;
            if (L.segLen[s] > *longest) *longest = L.segLen[s];
            for (int t = 0; t < L.segLen[s]; ++t) {
                const int cell = L.segCell[s] + t;
                ++covered[cell];
                const int shift = L.shifter[cell];
                const int row = shift >= 0 ? shift : L.shifter[cell + shift];
                const int off = shift >= 0 ? 0 : -shift;
                const int jp = L.rowJP[row] + off, kp = L.rowKP[row] + off, jkp = L.rowJKP[row] + off;
                if (jp != L.segJP[s] + t || kp != L.segKP[s] + t || jkp != L.segJKP[s] + t) ++bad;
                if (cell + 1 >= n || jp + 1 >= n || kp + 1 >= n || jkp + 1 >= n) ++bad;
                if (L.wallMap[cell] != -1 && L.wallMap[cell] != -2) ++bad;
            }
        }
        for (int q : L.specialCells) ++covered[q];
        for (int q : L.rotorCells) ++covered[q];
        for (int q = 0; q < n; ++q)
            if ((L.wallMap[q] == -3) != (covered[q] == 0) || covered[q] > 1) ++bad;
    }
    return bad;
}
