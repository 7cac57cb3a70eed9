/* CPU restatement of the CUDA-ORB detect / describe / match path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the sm_100a library, never the
 * product.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may load it.  Parity pinning: its outputs are compared against the
 * reference CUDA build itself (tests/golden/*.npz, produced by
 * tests/golden/make_golden.py from oracle/_ref/libref_orb.so on a B200).
 *
 * Memory model: pyramids use the reference layout (orb.cpp:145-191): octaves
 * stored back to back, pitch = align_up(width, 128).  Callers pass a pointer to
 * octave 0 inside a buffer that has at least ORACLE_GUARD zeroed bytes before
 * it and after the last octave, because the reference reads a little outside
 * each octave (orbd.cu:651-669, 1001-1036, 1437-1468).
 */
#ifndef ORB_ORACLE_H
#define ORB_ORACLE_H
#include <stdint.h>

#define ORACLE_GUARD (256 * 1024)

typedef struct {
  int x, y, octave;
  float score, angle;
  int match, distance;
} oo_point; /* same 28-byte layout as orb::OrbPoint (orb_structures.h:8-17) */

/* oszp = [osizes | widths | heights | pitchs | offsets(n+1)], as orb.cpp:151-156. */
int oo_layout(int w, int h, int noctaves, int* oszp);
void oo_fast_lut(int threshold, uint8_t* lut512);
void oo_umax(int patch_size, int* umax);
void oo_gauss_kernel(float* k4);
float oo_harris_scale(void);
int oo_pattern(int patch_size, int wta_k, int* pattern_xy);
float oo_fast_atan2(float y, float x);

void oo_pyramid(const uint8_t* img, int pitch_in, uint8_t* pyr, const int* oszp, int n);
void oo_score_map(const uint8_t* pyr, const int* oszp, int n, int threshold, int harris, int harris_fma,
                  float* vmap, int* layer);
int oo_nms(const float* vmap, const int* layer, const int* oszp, int n, int border, oo_point* out, int cap);
void oo_angle(const uint8_t* pyr, const int* oszp, int n, oo_point* pts, int npts, int patch_size);
void oo_blur(const uint8_t* pyr, uint8_t* out, const int* oszp, int n, int fma_h, int fma_v);
void oo_describe(const uint8_t* blurred, const int* oszp, int n, const oo_point* pts, int npts, const float* sinv,
                 const float* cosv, const int* pattern_xy, int wta_k, int rot_x, int rot_y, uint8_t* desc);
void oo_match(const uint8_t* d1, int n1, const uint8_t* d2, int n2, int* match, int* dist);
void oo_knn2(const uint8_t* q, int nq, const uint8_t* db, int ndb, uint32_t* dist2, int32_t* idx2);
int oo_threads(void);

/* FP64 side-oracle (Harris combine and angle polynomial in double) and the
 * per-keypoint exception flags of the parity report. */
#define ORACLE_TIE 1
#define ORACLE_STRADDLE_ANGLE 2
#define ORACLE_STRADDLE_DESC 4
void oo_harris_f64(const uint8_t* pyr, const int* oszp, int n, const oo_point* pts, int npts, double* score,
                   double* terms);
void oo_angle_f64(const uint8_t* pyr, const int* oszp, int n, const oo_point* pts, int npts, int patch_size,
                  double* angle);
void oo_exception_flags(const int* oszp, int n, const oo_point* pts, int npts, const float* sinv, const float* cosv,
                        const int* pattern_xy, int npat, int patch_size, double tie_eps, int* flags);
#endif
