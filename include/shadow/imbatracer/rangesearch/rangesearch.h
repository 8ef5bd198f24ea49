/* Include-path replacement for the reference's src/imbatracer/rangesearch/rangesearch.h.
 * Compile the reference with -I<this repository>/include/shadow -I<this repository>/include
 * ahead of its own src/ and link libimbart: every HashGrid<Iter, Photon> it declares — the
 * photon grid of LightVertices (light_vertices.h:70-100, used by VCMIntegrator's merging,
 * vcm.cpp:571-576) — is then libimbart's GPU grid behind the same build / query methods, with
 * no change to the reference's sources. The guard is the reference header's own, so a later
 * include of the original is skipped. */
#ifndef IMBA_RANGESEARCH_H
#define IMBA_RANGESEARCH_H

#include "imbart_hashgrid.hpp"

namespace imba {
template <typename Iter, typename Photon>
using HashGrid = ::imbart::GpuHashGrid<Iter, Photon>;
}

#endif
