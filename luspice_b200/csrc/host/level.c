/* Level (wave) sets of the static pattern: the rule of src/level.c:20-48.
 * Off-diagonal rows j of U(:,k) with 0 <= j < k are the columns column k
 * waits for; the diagonal is the last entry of each U column. */
#include <string.h>

#include "level.h"

int dsh_level_compute(int n, const int *Up, const int *Ui, int *level_out, int *nlevels_out)
{
    if (n < 0 || !Up || !Ui || !level_out || !nlevels_out) return 3;
    int deepest = 0;
    for (int k = 0; k < n; k++) {
        int lk = 0;
        for (int p = Up[k]; p < Up[k + 1] - 1; p++) {
            int j = Ui[p];
            if (j >= 0 && j < k && level_out[j] + 1 > lk) lk = level_out[j] + 1;
        }
        level_out[k] = lk;
        if (lk > deepest) deepest = lk;
    }
    *nlevels_out = deepest + 1;
    return 0;
}

int dsh_level_hist(int n, const int *level, int nlevels, int *hist_out)
{
    if (nlevels < 0 || !hist_out) return 3;
    memset(hist_out, 0, (size_t)nlevels * sizeof(int));
    for (int k = 0; k < n; k++)
        if (level[k] >= 0 && level[k] < nlevels) hist_out[level[k]]++;
    return 0;
}
