/* Wall-texture builders on the periodic grid (see textures.c). */
#ifndef DNSLBM_TEXTURES_H
#define DNSLBM_TEXTURES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void tex_smooth(int nx, int ny, int nz, int8_t *flags);
void tex_longitudinal(int nx, int ny, int nz, int gap, int width, int8_t *flags);
void tex_transverse(int nx, int ny, int nz, int gap, int width, int8_t *flags);
void tex_posts(int nx, int ny, int nz, int gx, int wx, int gy, int wy, int8_t *flags);
void tex_riblets(int nx, int ny, int nz, int height, int spacing, int8_t *flags);

#ifdef __cplusplus
}
#endif
#endif
