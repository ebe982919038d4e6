// Launch interface of the work-queue cycle kernel of 16-colour systems
// (J1 plus J2 / J3 shells, isotropic): a whole cycle of every such system in
// one launch.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"

namespace pyro {

// One (system, replica): its chunks of kPassThreads cells, the dependency
// half-width in chunks, its progress counters, and the position of its
// chunks among those of its group.
struct GenWaveUnit {
  int sys, rep;       // system index, replica within the system
  int n_chunks, dep;  // chunks per pass, dependency half-width (chunks)
  int prog_off;       // first progress counter of the unit
  int chunk_begin;    // first chunk of the unit within its group's chunks of a pass
};

// Units whose sweeps run together (their spins stay in L2): all passes of the
// group's units, pass by pass, before the next group's.
struct GenWaveGroup {
  int unit_begin, n_units;
  int chunks;        // chunks per pass over all units of the group
  int chunk_prefix;  // chunks per pass of the groups before it: the group's first
                     // item is 16 (n_metro + n_or) x chunk_prefix
};

// Items are numbered group by group; within a group pass by pass (16 colour
// passes per sweep, n_metro Metropolis sweeps then n_or over-relaxation
// sweeps); within a pass unit by unit, the chunks of pass k of a unit
// starting at chunk dep * k (modulo its chunks), so an item's inputs were
// issued about a pass earlier. The item of pass k on chunk q of a unit waits
// (acquire, bounded by spin_limit polls) until the unit's progress counters
// of chunks q - dep .. q + dep count k completed passes, and releases its own
// chunk's counter after its stores. It only waits on items with smaller
// tickets, taken by CTAs that are running, so the launch always progresses;
// a wait that runs out sets *status = 1 and the waiting CTA returns.
struct GenWaveParams {
  PassParams pass;  // sys, spins, temperatures, counters, seed; sweep_off = cycle's first sweep
  const GenWaveUnit* units;
  const GenWaveGroup* groups;
  const int* chunk_unit;  // unit of each chunk of one pass, groups in order (chunk_prefix + b)
  int n_groups;
  int n_metro, n_or;
  unsigned int* queue;     // next ticket, zero at launch
  unsigned int* progress;  // one counter per (unit, chunk), zero at launch
  int* status;
  int n_items;
  unsigned int spin_limit;
  int stall_item;  // diagnostics: this item never reports completion (-1: none)
};

cudaError_t launch_gen_wave(const GenWaveParams& p, cudaStream_t st);

}  // namespace pyro
