/*
 * readdy_b200_output.h -- the output files of the reference's standalone
 * native harness: trajectory frames (XML, which the coordinate reader of
 * readdy_b200_inputs.h reads back, and PDB) and the RDF table (CSV).
 * Replaces lib/ReaDDyGPU_Cpp/outputHandler/outputHandler.cpp:
 * RDFOutputHandler (openOutputFile :19-37, writeOutput :39-56),
 * PDBTrajectoryOutputHandler (:79-110) and XMLTrajectoryOutputHandler
 * (openOutputFile :119-127, closeOutputFile :129-133, writeFrame :135-148).
 *
 * Differences from the reference, on purpose:
 *   - XML coordinates are written with 17 significant digits (the reference
 *     writes 3 decimals), so a frame read back is the state bit for bit and
 *     the trajectory serves as a restart file;
 *   - the closing tag of an XML trajectory is </traj> (the reference writes
 *     "<\traj>", a tab);
 *   - every call reports failure with a negative RDGPU_ERR_* code and a
 *     message in rdgpu_output_error(), where the reference returns 1.
 */
#ifndef READDY_B200_OUTPUT_H
#define READDY_B200_OUTPUT_H
#include <stdint.h>
#include "readdy_b200.h"
#ifdef __cplusplus
extern "C" {
#endif

#define RDGPU_TRAJ_XML 0   /* <traj> of <tplgy_coords stepId=...> frames      */
#define RDGPU_TRAJ_PDB 1   /* MODEL / ATOM / ENDMDL records                    */

typedef struct rdgpu_traj* rdgpu_traj_handle;

/* Opens (truncates) a trajectory file of the given format.  Replaces the
   handlers' openOutputFile (outputHandler.cpp:79-87, :119-127).              */
int rdgpu_traj_open(const char* path, int32_t format, rdgpu_traj_handle* out);

/* Appends one frame of n particles: xyz (3n doubles), types (n), ids (n
   particle ids for the XML id attribute; NULL writes 1..n as the reference
   does).  PDB frames carry step as the MODEL number.  Replaces writeFrame
   (outputHandler.cpp:94-110, :135-148).                                      */
int rdgpu_traj_write(rdgpu_traj_handle t, int64_t step, int64_t n, const double* xyz, const int32_t* types,
                     const int32_t* ids);

/* Closes the file (XML: writes </traj> first); the handle is freed even when
   the close fails.  Replaces closeOutputFile (outputHandler.cpp:89-91,
   :129-133).                                                                  */
int rdgpu_traj_close(rdgpu_traj_handle t);

/* Writes the RDF table: a header "d" and ",\tRDF(a,b)" per ordered type pair
   (a, b) of the n_types names, then one row per bin with its lower edge
   k * rmax / nbins and the values g[(a * n_types + b) * nbins + k] (for
   example from rdgpu_rdf_normalized).  Replaces RDFOutputHandler
   (outputHandler.cpp:19-56).                                                  */
int rdgpu_write_rdf_csv(const char* path, int32_t n_types, const char* const* names, int32_t nbins, double rmax,
                        const double* g);

/* Message of the last failed call of this header (thread-local).             */
const char* rdgpu_output_error(void);

#ifdef __cplusplus
}
#endif
#endif
