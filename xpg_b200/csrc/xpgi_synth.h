// Synthetic frame generator of the benchmark workloads (not part of XPG's interface: XPG reads recorded frames;
// this produces seeded device-resident wedges for sweeps whose stack does not fit in host memory).
#ifndef XPGI_SYNTH_H
#define XPGI_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int n;                                  /* spots rendered (entries of index, or the first n spots) */
    const int32_t *index;                   /* (n) spots rendered, as indices into the arrays below; NULL: 0..n-1 */
    const double *x, *y, *z;                /* predicted centre (pixels, frame coordinate) */
    const double *counts;                   /* photons of the whole reflection */
    const double *sig_t, *sig_r, *sig_z;    /* tangential / radial width (pixels), rocking width (frames) */
    double orgx, orgy;                      /* beam centre (radial direction of the spots) */
} XiSynthSpots;

typedef struct {
    double level, ramp, orgx, orgy, rmax;   /* level * (1 + ramp * r / rmax) counts per pixel */
} XiSynthBackground;

/* Frames first_frame .. first_frame + n_frames - 1 (1-based) into out (n_frames, ny, nx) uint32. */
int xi_synth_frames(const XiSynthSpots *spots, const XiSynthBackground *bg, int first_frame, int n_frames, int ny,
                    int nx, uint64_t seed, int gaps, uint32_t *out, void *stream);
const char *xi_synth_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
