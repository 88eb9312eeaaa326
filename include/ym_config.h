/* ym_config.h -- canonical text configurations of SU(2) and SU(3) lattices,
 * the exchange and checkpoint format of the engine.
 *
 * SU(2): the reference's YM-SU2-CONFIG-V1 (Lattice4::to_canonical_config /
 * from_canonical_config, reference/rust/src/lib.rs:587-694), byte for byte:
 *   YM-SU2-CONFIG-V1\n
 *   extents=N0,N1,N2,N3\n
 *   link_count=L\n
 *   then L lines "a0,a1,a2,a3\n", each component the 16 lower-case hex digits
 *   of its binary64 bits, links in the reference order site*4 + mu.
 * Encoding refuses a lattice whose largest |norm^2 - 1| exceeds 2e-12
 * (NonUnitSu2); decoding checks the header, the declared count against the
 * reference cap (LatticeTooLarge) before the body, every token's shape,
 * every link's unit norm (NonFiniteSu2Component / NonUnitSu2), and that the
 * text is exactly the canonical re-encoding (InvalidConfigurationEncoding).
 *
 * SU(3): YM-SU3-CONFIG-V1, the same layout with one line of 18 hex words
 * per link (the 3x3 matrix row-major, real then imaginary part of each
 * entry).  The reference has no SU(3) text format; this one follows the
 * SU(2) rules with the reference's SU(3) gate (Su3::from_checked_matrix,
 * su3.rs:241-252: NonFiniteMatrix, NonUnitaryMatrix, DeterminantNotOne at
 * 5e-12) on decode and encode, and the SU(3) lattice cap of 2^18 links
 * (su3_lattice.rs:17).
 *
 * lift_reference_caps != 0 lifts the link-count caps for lattices beyond the
 * reference's reach.  Links are host arrays in the reference layout: SU(2)
 * [links][4] binary64, SU(3) [links][3][3][2] binary64.  The encoders write
 * no terminating NUL; *length receives the byte count (pass text = NULL to
 * query it).  The decoders fill extents first; with links = NULL they stop
 * there, so a caller can size the link buffer.
 */
#ifndef YM_CONFIG_H
#define YM_CONFIG_H

#include <stdint.h>

#include "ym_status.h"

#ifdef __cplusplus
extern "C" {
#endif

#define YM_SU2_CONFIG_FORMAT_ID "YM-SU2-CONFIG-V1"
#define YM_SU3_CONFIG_FORMAT_ID "YM-SU3-CONFIG-V1"

int32_t ym_su2_to_canonical_config(const int64_t extents[4], const double *links,
                                   int32_t lift_reference_caps, char *text, int64_t capacity,
                                   int64_t *length);
int32_t ym_su2_from_canonical_config(const char *text, int64_t length, int32_t lift_reference_caps,
                                     int64_t extents[4], double *links, int64_t links_capacity);
int32_t ym_su3_to_canonical_config(const int64_t extents[4], const double *links,
                                   int32_t lift_reference_caps, char *text, int64_t capacity,
                                   int64_t *length);
int32_t ym_su3_from_canonical_config(const char *text, int64_t length, int32_t lift_reference_caps,
                                     int64_t extents[4], double *links, int64_t links_capacity);

#ifdef __cplusplus
}
#endif

#endif /* YM_CONFIG_H */
