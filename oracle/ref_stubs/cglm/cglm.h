/* Minimal stand-in for the cglm header the reference's initial-condition code
 * includes (initialConditions.h:9).  cglm is not installed here; the harness
 * never calls the initial-condition code, but it must compile and link.
 * Matrices are column-major like cglm's: m[column][row]. */
#ifndef REF_STUB_CGLM_H
#define REF_STUB_CGLM_H

typedef float vec3[3];
typedef float mat3[3][3];

#define GLM_PIf 3.14159265358979323846f

static inline void glm_mat3_mul(mat3 a, mat3 b, mat3 dest) {
    mat3 r;
    for (int c = 0; c < 3; c++)
        for (int row = 0; row < 3; row++)
            r[c][row] = a[0][row] * b[c][0] + a[1][row] * b[c][1] + a[2][row] * b[c][2];
    for (int c = 0; c < 3; c++)
        for (int row = 0; row < 3; row++) dest[c][row] = r[c][row];
}

static inline void glm_mat3_mulv(mat3 m, vec3 v, vec3 dest) {
    vec3 r;
    for (int row = 0; row < 3; row++) r[row] = m[0][row] * v[0] + m[1][row] * v[1] + m[2][row] * v[2];
    dest[0] = r[0];
    dest[1] = r[1];
    dest[2] = r[2];
}

#endif
