/*
 * level.h - level (wave) scheduling of the static L/U pattern.
 *
 * Drop-in for LUspice src/level.h:9-10.  level[k] = 1 + max level[j] over
 * the off-diagonal rows j < k of U(:,k) (0-based, columns with no such row
 * are level 0); *nlevels_out = max level + 1 (src/level.c:20-38).  Columns
 * of one level have no dependency on each other and are refactored
 * concurrently.
 */
#ifndef DSH_LEVEL_H
#define DSH_LEVEL_H

#ifdef __cplusplus
extern "C" {
#endif

int dsh_level_compute(int n, const int *Up, const int *Ui, int *level_out, int *nlevels_out);
int dsh_level_hist(int n, const int *level, int nlevels, int *hist_out);

#ifdef __cplusplus
}
#endif

#endif /* DSH_LEVEL_H */
