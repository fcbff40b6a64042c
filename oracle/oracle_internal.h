/*
 * oracle_internal.h — TEST INFRASTRUCTURE ONLY: geometry helpers shared by
 * the oracle's sources (triangle soups, ray maps, ray/triangle tests).
 */
#ifndef LBM_ORACLE_INTERNAL_H
#define LBM_ORACLE_INTERNAL_H

/* STLStruct (include/types.h:244-256): triangles as nine coordinate arrays,
 * bounds, and the spatial bins of sortSTLToBins. */
typedef struct ostl {
    int count;
    float *ax, *ay, *az, *bx, *by, *bz, *cx, *cy, *cz;
    float xMin, yMin, zMin, xMax, yMax, zMax;
    float binSize, oxBin, oyBin, ozBin;
    int binCountX, binCountY, binCountZ;
    int* firstInBin; /* [bins + 1] */
    int* bin;        /* triangle indices, grouped by bin */
} ostl;

/* RayMapStruct (include/types.h:166): per (i, j) ray the sorted hit list;
 * scan[ray] .. scan[ray + 1] index map[]. */
typedef struct oraymap {
    int nx, ny;
    long long* scan;
    int* map;
} oraymap;

int ostl_load(ostl* t, const float* tri, int n);
void ostl_bins(ostl* t, float resGlobal);
void ostl_free(ostl* t);

void oray_voxelize(oraymap* m, const ostl* t, float ox, float oy, float oz, float res, int nx, int ny);
void oray_union(oraymap* sum, const oraymap* bonus);
void oray_copy(oraymap* dst, const oraymap* src);
void oray_empty(oraymap* m, int nx, int ny);
void oray_free(oraymap* m);
int oray_solid(const oraymap* m, int i, int j, int k);
int oray_block_has_fluid(const oraymap* m, int ic, int jc, int kc, int down);
int oray_block_has_wall(const oraymap* m, int ic, int jc, int kc, int down);
int oray_triangle(float ax, float ay, float az, float bx, float by, float bz, float cx, float cy, float cz, float ex,
                  float ey, float ez, float edgeTol, float* tOut);

#endif
