/*
 * pyro.h — C-ABI of the B200 Monte Carlo engine for classical O(3)
 * Heisenberg spins on the pyrochlore lattice (16 L^3 sites, 6 nearest
 * neighbours; H = J1 sum_<ij> S_i.S_j + J2 sum_<<ij>> + J3 sum_<<<ij>>>).
 *
 * It replaces the host interface of taillefu/cudacode, whose functions all
 * return void, print and exit() on error, and keep their state in a
 * `std::vector<dev>`. Here every call returns an int status (PYRO_OK or a
 * negative PYRO_ERR_* code, with a message from pyro_last_error()), all device
 * state lives in an opaque pyro_ctx (one per GPU), and the caller owns every
 * host array it passes. Calls are stream-ordered on the context's stream and
 * return without waiting, except those that copy results to host memory.
 * A context is not thread-safe; use one context per GPU and per thread.
 *
 * Spin layout (device and host): per system, per replica, 16 planes (one per
 * site of the conventional cubic cell, s = 4 f + b with f the FCC corner and b
 * the pyrochlore sublattice), each plane L^3 cells with cell = (z L + y) L + x;
 * one float4 (x, y, z, 0) per spin.
 */
#ifndef PYRO_H
#define PYRO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PYRO_OK 0
#define PYRO_ERR_ARG -1      /* invalid argument or configuration        */
#define PYRO_ERR_CUDA -2     /* a CUDA runtime call failed               */
#define PYRO_ERR_TIMEOUT -3  /* a bounded device wait ran out            */
#define PYRO_ERR_NAN -4      /* non-finite or non-unit spins detected    */
#define PYRO_ERR_IO -5       /* checkpoint file missing, short or corrupt */
#define PYRO_ERR_STATE -6    /* call not valid in the current state       */
#define PYRO_ERR_NOMEM -7    /* device allocation failed                 */

/* One lattice with its own size, couplings and temperature ladder. */
typedef struct {
  int L;                      /* cubic cells per edge (>= 2)                       */
  int n_replicas;             /* replicas held by this context                     */
  int replica_offset;         /* global index of the first one (sharding over GPUs) */
  int n_temperatures;         /* full ladder size; == n_replicas when not sharded   */
  const double* temperatures; /* n_temperatures values, strictly increasing          */
  double J1;                  /* nearest neighbour (distance sqrt(2)/4 a)            */
  double J2;                  /* second neighbour (sqrt(6)/4 a)                      */
  double J3;                  /* third neighbour through a site (sqrt(2)/2 a, J3a)   */
  double J3b;                 /* third neighbour across a hexagon (sqrt(2)/2 a)      */
} pyro_system_desc;

typedef struct {
  int n_systems;
  const pyro_system_desc* systems;
  uint64_t seed;     /* Philox key; all randomness is a function of (seed, counters) */
  int device;        /* CUDA device ordinal                                         */
  int renorm_every;  /* renormalise spins every this many sweeps (0 = never)        */
} pyro_config;

typedef struct pyro_ctx pyro_ctx;

/* Context life cycle. Replaces InitializeDevice + InitializeCouplings3D
 * (Pyrochlore.cu:643-711, 1251-1267). */
int pyro_create(const pyro_config* cfg, pyro_ctx** out);
int pyro_destroy(pyro_ctx* ctx);
const char* pyro_last_error(const pyro_ctx* ctx);
int pyro_version(void);
/* Host-only: the neighbour table of cubic-cell site `site` (0..15) in the
 * canonical order (J1 6, J2 12, J3a 6, J3b 6): out[4k..4k+3] = dx, dy, dz,
 * target site. Replaces the packed links16 table of InitializeCouplings3D
 * (Pyrochlore.cu:152-167, 643-711). Needs no GPU. */
int pyro_neighbour_table(int site, int* out120);

/* Kernel choices (the autotuner's knobs). PYRO_OPT_J1_KERNEL: 1 (default)
 * runs J1-only systems on the specialised one-thread-per-cell kernels, 0 on
 * the generic colour-pass kernel; results are bit-identical either way. */
#define PYRO_OPT_J1_KERNEL 1
/* PYRO_OPT_CYCLE_KERNEL: 1 sweeps J1-only systems with the
 * cluster-resident kernel (one thread-block cluster per replica runs every
 * colour pass of a call, so the replica stays in L2), 0 (default) with one
 * launch per colour pass. 2 runs the colour passes of a pyro_cycle (and its
 * energies) of each J1 system as one launch over a work queue: an item is
 * one pass of a 256-cell chunk of one replica, items are numbered replica
 * group (PYRO_OPT_REPLICA_GROUP, 0 = all replicas) by replica group and pass
 * by pass, and each item waits only until the previous pass is complete on
 * the chunks that hold its neighbours (per-chunk counters, released and
 * acquired at GPU scope, every wait bounded; a wait that runs out makes the
 * next pyro_synchronize return PYRO_ERR_TIMEOUT). PYRO_OPT_J1_SITE_MODE
 * chooses its pass forms. With 2, when every other system is an isotropic
 * 16-colour system (J2 or J3 set), their sweeps of a pyro_cycle run as one
 * more work-queue launch over all of them: units (system, replica) in
 * groups of about PYRO_OPT_GROUP_MB MB (0: one group), items of one 16-colour
 * pass of a 256-cell chunk, the same waits and bounds; their energies come
 * from the observables kernel after it. 3 runs them as skewed launches: replica group g
 * (PYRO_OPT_REPLICA_GROUP replicas, 0 = 2) runs its pass k in launch
 * s g + k, with s chosen so that about PYRO_OPT_CHAINS groups are in flight
 * in every launch; a launch's items belong to different replicas and need
 * no synchronisation, and its groups' spins stay in L2. Calls other than
 * pyro_cycle use the per-pass kernels. PYRO_OPT_CLUSTER_SIZE: CTAs per cluster (2, 4, 8, 16; the
 * context falls back to the largest size that can be resident).
 * Identical results in every mode. */
#define PYRO_OPT_CYCLE_KERNEL 2
#define PYRO_OPT_CLUSTER_SIZE 3
/* PYRO_OPT_J1_SITE_MODE: bit 0 = Metropolis passes, bit 1 = over-relaxation
 * passes of the per-pass J1 kernel run one site per thread (set) or the four
 * sites of a cell per thread (clear). Default 1. */
#define PYRO_OPT_J1_SITE_MODE 4
/* PYRO_OPT_SMEM_KERNEL: 1 (default) runs pyro_cycle without exchange, when
 * every system has L <= 8, as one launch per system with each replica held
 * in one CTA's shared memory for all cycles; 0 uses the other kernels.
 * Identical results. */
#define PYRO_OPT_SMEM_KERNEL 5
/* PYRO_OPT_REPLICA_GROUP: with the per-pass J1 kernels, run every sweep of
 * one group of this many replicas before the next group (0, default: all
 * replicas in every pass), keeping a group's spins in L2. Identical results. */
#define PYRO_OPT_REPLICA_GROUP 6
/* PYRO_OPT_CHAINS: 1..8 concurrent streams (parallel branches of the cycle
 * graph) the replica groups are dealt to; with PYRO_OPT_CYCLE_KERNEL 3, the
 * replica groups in flight in one launch. Identical results. */
#define PYRO_OPT_CHAINS 7
/* PYRO_OPT_GROUP_MB: run the generic (J2/J3) colour passes over groups of
 * replicas of about this many MB, all sweeps of a group before the next,
 * groups dealt to the PYRO_OPT_CHAINS streams (0, default: off).
 * Identical results. */
#define PYRO_OPT_GROUP_MB 8
/* PYRO_OPT_FAR_KERNEL: 1 (default) runs 16-colour passes (J2/J3 systems) on
 * the kernel with compile-time neighbour offsets, 0 on the generic kernel.
 * Identical results. */
#define PYRO_OPT_FAR_KERNEL 9
/* PYRO_OPT_PDL: 1 (default) launches the per-pass kernels (nearest-neighbour,
 * 16-colour and generic)
 * with programmatic dependent launch, so a pass's launch overlaps the drain
 * of the previous kernel in its stream (each pass waits for that kernel's
 * completion before touching memory: results are unchanged); 0 plain
 * launches. */
#define PYRO_OPT_PDL 10
/* PYRO_OPT_TET_GROUPED: 1 (default) runs the learned tetrahedron sweeps of
 * pyro_cycle_tet inside the replica groups of PYRO_OPT_REPLICA_GROUP, each
 * group's right after its plain sweeps on the same chain; 0 runs them over
 * all replicas after every group's plain sweeps. Identical results. */
#define PYRO_OPT_TET_GROUPED 11
/* PYRO_OPT_FUSED_OBS: 1 (default) computes the FP64 energy and magnetisation
 * of an isotropic J1 replica group inside the group's last colour pass of a
 * cycle (when that pass runs one cell per thread), from the spins the pass
 * has just loaded; 0 runs a separate observables kernel after the pass.
 * Same spins; energies equal up to FP64 summation order. */
#define PYRO_OPT_FUSED_OBS 12
/* PYRO_OPT_WAVE_STALL (diagnostics of the work-queue cycle kernel): when
 * >= 0, item `value` of the kernel's launches never reports its completion
 * and every dependency wait gives up after 4096 polls, so the cycle ends
 * with its waits run out: the next pyro_synchronize returns
 * PYRO_ERR_TIMEOUT (and clears the condition) and the spins are left
 * partly updated. -1 (default) is normal operation. Used to test the
 * bounded waits without a device fault. */
#define PYRO_OPT_WAVE_STALL 13
/* PYRO_OPT_MEASURE_SNAPSHOT: 1 makes the measurement calls
 * (pyro_last_observables, pyro_get_temperatures, pyro_get_permutation,
 * pyro_order_parameters, pyro_sublattice_magnetisation,
 * pyro_structure_factor, pyro_ising_configuration) read the last
 * pyro_snapshot on the context's measurement stream, so they run while the
 * Monte Carlo calls queued after the snapshot proceed on the context
 * stream; 0 (default) reads the live state on the context stream. Needs a
 * snapshot first (else PYRO_ERR_STATE). Changes no kernel schedule. */
#define PYRO_OPT_MEASURE_SNAPSHOT 14
/* PYRO_OPT_J1_FIXED_L: 1 (default) runs the per-pass kernels of isotropic
 * J1 systems with L = 16 or 32 in forms compiled for that L (cell decode by
 * shifts, neighbour planes as compile-time offsets: fewer instructions per
 * update); 0 uses the run-time-L kernels for every L. Identical results. */
#define PYRO_OPT_J1_FIXED_L 15
/* PYRO_OPT_CHAIN_STAGGER: with replica groups on PYRO_OPT_CHAINS > 1
 * chains, each odd chain c starts its first group after chain c - 1 has run
 * its first `value` colour passes (at most one group's; 0, default: all
 * chains start together), so the Metropolis phases of a chain pair do not
 * coincide. Identical results. */
#define PYRO_OPT_CHAIN_STAGGER 16
int pyro_set_option(pyro_ctx* ctx, int option, int value);
int pyro_get_option(pyro_ctx* ctx, int option, int* value);
/* Autotuner: times every kernel variant (per-pass generic, per-pass J1,
 * per-pass J1 in its site/cell forms, replica groups of 1..8 on 1..8
 * concurrent chains, cluster-resident J1 with cluster sizes 16, 10, the
 * work-queue cycle kernel in its forms over replica groups of 2..16 or all) on
 * `cycles` cycles of n_metro + n_or sweeps (+ exchange when the context holds
 * the whole ladder) and keeps the fastest; *chosen = its index. The timed
 * cycles are real Monte Carlo steps and advance the chain. */
int pyro_autotune(pyro_ctx* ctx, int n_metro, int n_or, int cycles, int* chosen);

/* Stream used by every call (default: a stream the context creates). */
int pyro_set_stream(pyro_ctx* ctx, void* cuda_stream);
void* pyro_get_stream(const pyro_ctx* ctx);
/* Wait for all work queued by the context. Replaces SynchronizeJobs
 * (MonteCarlo.cu:230-245). */
int pyro_synchronize(pyro_ctx* ctx);
/* Philox keys of one system: its replica r draws with the replica word
 * key_base + replica_offset + r and its exchanges with the word swap_key.
 * By default key_base is the number of temperatures of the systems before it
 * in the context and swap_key its index, so that no two systems share a
 * stream; a context holding a subset of a larger set of independent systems
 * (one rank's share, see cudacode_b200/distributed.py) sets each system's
 * keys to those it has in the full set and reproduces its chain bit for
 * bit. Synchronises the context stream; drops the captured cycles. */
int pyro_set_system_keys(pyro_ctx* ctx, int system, int key_base, int swap_key);
/* Measurement snapshot. Replaces ExtractConfigurationsFromMonteCarlo
 * (Pyrochlore.cu:1608-1617), which copies the working spins into a
 * measurement buffer so that the next Monte Carlo block runs while the
 * previous one is measured (ApplyParallelTemperingDuringMeasure,
 * MonteCarlo.cu:613-657). Queues, at the current point of the context
 * stream, a device copy of every system's spins, of the replica <->
 * temperature maps and of the last cycle's FP64 energies and
 * magnetisations, on the context's measurement stream; the context stream's
 * next work waits only for that copy (a few hundred microseconds for
 * gigabytes of spins). Returns without waiting; the first call allocates the
 * snapshot buffers. Not allowed during a stream capture. */
int pyro_snapshot(pyro_ctx* ctx);

/* Sizes of one system, and the number of colour classes its sweep uses
 * (4 for J1 only, 16 when J2/J3 are present). */
int pyro_system_info(const pyro_ctx* ctx, int system, int* L, int* n_sites,
                     int* n_replicas, int* n_colours);

/* Spins. Uniform random unit vectors from Philox(seed; site, replica):
 * replaces GenerateRandomVectorsOnDevice / Generate3DVectorList
 * (MonteCarlo.cu:257-293, Math.cu:132-143). set/get copy one system's
 * replicas in the float4 layout above; replace the configuration transfers
 * of Save/ReadConfigurations (Math.cu:618-701). */
int pyro_init_random(pyro_ctx* ctx);
int pyro_set_spins(pyro_ctx* ctx, int system, const float* host_xyzw);
int pyro_get_spins(pyro_ctx* ctx, int system, float* host_xyzw);
/* The same in the reference's spin layout (Sx = spin + 3 Offset, Sy = Sx +
 * 16 L^3, Sz = Sy + 16 L^3, Pyrochlore.cu:288-290 with Offset = replica x
 * 16 L^3, Math.cu:93): per replica three planes x, y, z of 16 L^3 doubles
 * (site index s L^3 + cell), replicas consecutive; values are rounded to
 * FP32 on the way in. Synchronous. */
int pyro_set_spins_planar(pyro_ctx* ctx, int system, const double* host_planes);
int pyro_get_spins_planar(pyro_ctx* ctx, int system, double* host_planes);
/* Device-pointer variants (stream-ordered; the pointer must hold one system). */
int pyro_set_spins_device(pyro_ctx* ctx, int system, const float* dev_xyzw);
int pyro_get_spins_device(pyro_ctx* ctx, int system, float* dev_xyzw);

/* Plain method. One sweep = every colour class in order, each updated in
 * one pass. Metropolis uses a cone proposal of half-angle acos(cosmax[t]) of
 * the replica's temperature slot t. Replaces Mc / MCMultipleTemperaturesPerSystem
 * (Pyrochlore.cu:74-133, 829-885) and OverRelaxationByPiStep (975-1007). */
int pyro_metropolis_sweep(pyro_ctx* ctx, int n_sweeps);
int pyro_overrelax_sweep(pyro_ctx* ctx, int n_sweeps);

/* Cone widths (cos of the half-angle) per temperature slot of one system,
 * and acceptance counts since the last reset. Replace CosThetaSolid and
 * CalculateRatio (MonteCarlo.cu:346-367). */
int pyro_set_cone(pyro_ctx* ctx, int system, const float* cosmax);
int pyro_get_cone(pyro_ctx* ctx, int system, float* cosmax);
int pyro_get_acceptance(pyro_ctx* ctx, int system, uint64_t* accepted, uint64_t* proposed);
int pyro_reset_acceptance(pyro_ctx* ctx);
/* Adapt each temperature's cone to `target` acceptance with `iterations`
 * rounds of `sweeps_per_iteration` Metropolis sweeps (+ n_or over-relaxation
 * sweeps each). Replaces CalculateSolidAngle (MonteCarlo.cu:371-426). */
int pyro_tune_cone(pyro_ctx* ctx, double target, int iterations, int sweeps_per_iteration,
                   int n_or);

/* FP64 energy and magnetisation per replica of one system (replica order,
 * i.e. configuration slots, not temperature order). Synchronous. Replaces
 * TotalEnergyv2 (Math.cu:309-330) and Magnetization (Pyrochlore.cu:453-466). */
int pyro_observables(pyro_ctx* ctx, int system, double* energy, double* magnetisation3);
/* Stream-ordered variant into device buffers (n_replicas and 3 n_replicas). */
int pyro_observables_device(pyro_ctx* ctx, int system, double* dev_energy,
                            double* dev_magnetisation3);
/* The energies / magnetisations of the last pyro_cycle (computed at the end
 * of every cycle without learned moves) or pyro_observables* call, copied to
 * device memory without recomputing them (replica order, stream-ordered). */
int pyro_last_observables_device(pyro_ctx* ctx, int system, double* dev_energy,
                                 double* dev_magnetisation3);
/* The same to host memory (synchronous). */
int pyro_last_observables(pyro_ctx* ctx, int system, double* energy, double* magnetisation3);

/* Stream-ordered forms with host buffers, for drivers that queue the next
 * step before reading the last one: the copy is queued on the context's
 * stream and the call returns at once. The buffers must be pinned host
 * memory (cudaHostAlloc or cudaHostRegister; else PYRO_ERR_ARG); the cone
 * widths are checked when the call is made and must not change, and the
 * observables must not be read, until pyro_synchronize has returned. Not in
 * the PYRO_OPT_MEASURE_SNAPSHOT mode (PYRO_ERR_STATE). */
int pyro_set_cone_async(pyro_ctx* ctx, int system, const float* pinned_cosmax);
int pyro_last_observables_async(pyro_ctx* ctx, int system, double* pinned_energy,
                                double* pinned_magnetisation3);

/* Temperatures. temperature_of_replica: T of each configuration slot (the
 * reference's permuted `Temperatures` vector); replica_of_temperature: the
 * inverse map. Global indices (all n_temperatures entries). */
int pyro_get_temperatures(pyro_ctx* ctx, int system, double* temperature_of_replica);
int pyro_get_permutation(pyro_ctx* ctx, int system, int* replica_of_temperature);

/* Replica exchange between neighbouring temperatures (pairs (t, t+1) with
 * t % 2 == parity), FP64 test, Philox(seed; pair, swap count). The temperature
 * labels move, spins stay. Replaces TrySwapingTemperatures
 * (MonteCarlo.cu:105-172). parity < 0 alternates automatically.
 * n_accepted may be NULL (then the call does not synchronise). */
int pyro_pt_swap(pyro_ctx* ctx, int parity, int* n_accepted);
/* Sharded form: energies of ALL n_temperatures replicas of `system` (global
 * replica order, device memory), gathered by the caller across GPUs. Every
 * rank applies the identical decision. */
int pyro_pt_swap_global(pyro_ctx* ctx, int system, const double* dev_energy_all, int parity);
int pyro_get_swap_stats(pyro_ctx* ctx, int system, uint64_t* accepted, uint64_t* attempted);

/* One or more cycles of n_metro Metropolis + n_or over-relaxation sweeps,
 * energy, and (if do_swap) a replica exchange of alternating parity, replayed
 * from a CUDA graph. Replaces ParallelTempering (MonteCarlo.cu:429-470).
 * If a history buffer is enabled, each cycle appends the energy of every
 * temperature slot. */
int pyro_cycle(pyro_ctx* ctx, int n_metro, int n_or, int do_swap, int n_cycles);
int pyro_enable_history(pyro_ctx* ctx, int capacity_cycles);
/* Copies min(capacity, recorded) cycles of system `system`: out[c * n_temperatures + t]. */
int pyro_get_history(pyro_ctx* ctx, int system, double* out, int* n_cycles);

/* Counters: sweeps done so far (all systems advance together), and kernels
 * launched by pyro_cycle / pyro_cycle_tet (graph replays count the kernels
 * of the captured graph). */
int pyro_get_sweep_count(pyro_ctx* ctx, uint64_t* sweeps);
int pyro_get_launch_count(pyro_ctx* ctx, uint64_t* launches);

/* Check that every spin is finite with |S|^2 within tol of 1; returns
 * PYRO_ERR_NAN and the first bad spin index otherwise. */
int pyro_check_spins(pyro_ctx* ctx, float tol, long long* first_bad);

/* Checkpoint / resume: the whole chain state (spins, temperature labels,
 * cone widths, sweep and exchange counters, learned-move weights and
 * counter) in one file with a checksum. Philox is counter-based, so this is
 * all a resumed run needs to continue bit for bit. Loading into a context
 * created with another configuration gives PYRO_ERR_ARG; a missing, short
 * or corrupt file PYRO_ERR_IO (nothing is changed then). Replaces the
 * InitialConf%d.dat / Conf%d.dat files and --ContinueMeasurement of the
 * reference (Math.cu:618-701, Pyrochlore.cu:1190-1194, 1528-1531). */
int pyro_save_checkpoint(pyro_ctx* ctx, const char* path);
int pyro_load_checkpoint(pyro_ctx* ctx, const char* path);
/* The reference's configuration files (SaveConfigurations /
 * ReadConfigurations, Math.cu:618-701): "<prefix><k>.dat" per temperature,
 * k = 0 the highest, each repetition the spins as consecutive (x, y, z)
 * doubles in site-plane-then-cell order; save appends a repetition if
 * `append`, read loads repetition `repetition` into the replica that holds
 * each temperature. */
int pyro_save_configurations(pyro_ctx* ctx, int system, const char* prefix, int append);
int pyro_read_configurations(pyro_ctx* ctx, int system, const char* prefix, int repetition);

/* Bond-dependent nearest-neighbour exchange and Zeeman field of one system
 * (the reference's anisotropic model: bond matrices couplings_const,
 * Pyrochlore.cu:169-184, used by CalculateLocalExchangeField 210-275 and
 * TotalEnergy 468-523; site fields InitializeMagneticField 414-450):
 *   H = sum_<ij> S_i^T A[b_i][b_j] S_j - sum_i f[b_i] . S_i + (J2, J3 shells),
 * S unit vectors, b = site & 3 the pyrochlore sublattice.
 * exchange144[(4 a + b) * 9 + 3 r + c] = A[a][b][r][c]; A[b][a] must be the
 * transpose of A[a][b] (else PYRO_ERR_ARG); the diagonal blocks are ignored.
 * field12[3 b + r] = f[b][r] (NULL: no field). The matrices replace the
 * system's J1; its J2 / J3 shells stay. exchange144 = NULL returns the
 * system to isotropic J1. Updates keep the bit-exact contract (each bond one
 * pyro_matvec_add in canonical neighbour order, then minus f). Such a system
 * runs on the generic and shared-memory kernels; the learned tetrahedron
 * move skips it. Invalidates the captured cycle graphs. */
int pyro_set_exchange(pyro_ctx* ctx, int system, const double* exchange144,
                      const double* field12);
/* The system's matrices and field as set (is_set = 0 for isotropic J1). */
int pyro_get_exchange(pyro_ctx* ctx, int system, double* exchange144, double* field12,
                      int* is_set);
/* The reference's parameterisation in this convention, so that energies
 * and temperatures equal the reference's (its spin-1/2 factor 1/4 folded
 * in): A = -C / 4 with C the couplings_const matrices of J1..J4
 * (Pyrochlore.cu:169-184), generated from the lattice symmetry; and
 * f_b = (1/2) mu_B g_b B with g_b = gxy I + (gz - gxy) z_b z_b^T (z_b the
 * local <111> axis of sublattice b), B in tesla, mu_B = 0.0578838261305
 * meV/T (InitializeMagneticField, Pyrochlore.cu:414-450). */
int pyro_reference_exchange(double J1, double J2, double J3, double J4, double* exchange144);
int pyro_reference_field(double gxy, double gz, const double* B3, double* field12);
/* The reference's g-tensors g_b = gxy I + (gz - gxy) z_b z_b^T of the four
 * sublattices, g36[9 b + 3 r + c] (MagnetizationGPU, Pyrochlore.cu:277-342,
 * InitializeMagneticField 414-450). */
int pyro_reference_gtensor(double gxy, double gz, double* g36);
/* FP64 magnetisation of each sublattice of every replica held (replica
 * order), out[(r * 4 + b) * 3 + k] = sum of S^k over the sites of
 * sublattice b; the reference's g-weighted moment of MagnetizationGPU
 * (Pyrochlore.cu:277-342) is sum_b g_b m_b. Synchronous. */
int pyro_sublattice_magnetisation(pyro_ctx* ctx, int system, double* out);

/* Order parameters of every replica held (replica order), FP64 sums over
 * the lattice, out[r * 20 + q]:
 *   q = 0..11  irrep components of Measurement (Pyrochlore.cu:526-641):
 *              A2, E (2), T (3), uniform magnetisation (3), T' (3);
 *   q = 12..17 quadrupole sum (S^a S^b - delta_ab/3), ab = xx xy xz yy yz zz
 *              (_CudaQuadrupolarOrder, Math.cu:335-372);
 *   q = 18     monopole density, sum over cells of 1/4 sum over its four
 *              up-tetrahedra of |sum_b a_b . S| (CudaCalculateMonopoleSquare,
 *              Math.cu:386-476);
 *   q = 19     sum |a_b . S| / sqrt 3 (CudaCalculateAbsSz, Math.cu:478-510);
 * a_b = (1,1,1), (-1,-1,1), (1,-1,-1), (-1,1,-1). Synchronous. */
int pyro_order_parameters(pyro_ctx* ctx, int system, double* out);
/* Ising projection of one replica (CudaCalculateIsingConf, Math.cu:513-541):
 * out[cell] (L^3 ints) has bit 4 t + b set where a_b . S < 0 for the site
 * 4 t + b of the cell. Synchronous. */
int pyro_ising_configuration(pyro_ctx* ctx, int system, int replica, int* out);

/* Static structure factor S(q) = (1/N) sum_a |sum_i S_i^a e^{-i q.r_i}|^2,
 * averaged over the replicas held, on a grid of G^3 wave vectors
 * q = (2 pi / L) * stride * (h, k, l), h, k, l in [-G/2, G/2); out[(h' G + k') G + l'].
 * One replica `replica` (>= 0) or all (-1). Replaces the cuFFT-based
 * StructFactor path (Math.cu:721-741, Pyrochlore.cu:1303-1419). */
int pyro_structure_factor(pyro_ctx* ctx, int system, int replica, int G, int stride, double* out);

/* Learned tetrahedron proposal (no counterpart in the reference).
 * Up-tetrahedra of one FCC corner share no bond, so the four corners are four
 * colour classes; a tetrahedron sweep is one pass per class. For each
 * up-tetrahedron a 16 -> 64 -> 64 -> 16 MLP (BF16 weights, FP32 tensor-core
 * accumulation) maps the external fields of its four spins and beta to a
 * von Mises-Fisher distribution per spin; a joint move drawn from it is
 * accepted with the exact Metropolis-Hastings ratio (FP32 energy of the
 * tetrahedron), so detailed balance holds for any weights. J1-only systems.
 *
 * pyro_tet_init: allocates the network (He-initialised from `seed`) and a ring
 * of `sample_capacity` training samples. Weights: 6288 FP32 values, layout
 * W1[16][64], b1[64], W2[64][64], b2[64], W3[64][16], b3[16] (row = input). */
int pyro_tet_init(pyro_ctx* ctx, uint64_t seed, long long sample_capacity);
int pyro_tet_set_weights(pyro_ctx* ctx, const float* weights, int n);
int pyro_tet_get_weights(pyro_ctx* ctx, float* weights, int n);
/* n learned tetrahedron sweeps of every J1-only system. */
int pyro_tet_sweep(pyro_ctx* ctx, int n_sweeps);
/* 0: one launch per corner pass, one lane per tetrahedron; 1: all passes of
 * a call in one launch, one thread-block cluster per replica; 2 (default):
 * one launch per corner pass, two lanes per tetrahedron (0, 1 and 2 give
 * identical results); 3: one launch per corner pass with the network on the
 * 5th-generation tensor cores (tcgen05.mma, accumulators in tensor memory),
 * 128 tetrahedra per CTA: the same move, with its own rounding of the
 * network's accumulations. A tensor-core wait that runs out in form 3 skips
 * the moves of its CTA and makes pyro_tet_acceptance return
 * PYRO_ERR_TIMEOUT. */
int pyro_tet_set_kernel(pyro_ctx* ctx, int mode);
/* Proposal of the learned move. 1 (default): sites 0-2 of the tetrahedron
 * from the network's vMFs, site 3 from its exact conditional distribution
 * given the three proposed spins and its external field, a vMF of natural
 * parameter -beta (J1 (s0' + s1' + s2') + h3); 0: all four sites from the
 * network's vMFs. Both are exact MH moves. */
int pyro_tet_set_proposal(pyro_ctx* ctx, int kind);
int pyro_tet_acceptance(pyro_ctx* ctx, int system, uint64_t* accepted, uint64_t* proposed);
int pyro_tet_reset_acceptance(pyro_ctx* ctx);
/* Appends (features[16], spins[12]) of every stride-th up-tetrahedron of each
 * class and replica of `system` to the sample ring (oldest overwritten). */
int pyro_tet_collect(pyro_ctx* ctx, int system, int stride, long long* n_written);
int pyro_tet_samples(pyro_ctx* ctx, float* features, float* targets, long long max_n,
                     long long* n_out);
/* `steps` Adam steps (lr, beta 0.9/0.999) of maximum likelihood on random
 * batches of `batch` samples; *mean_loss (may be null) = last batch's mean
 * negative log-likelihood. Returns after the context stream has drained. */
int pyro_tet_train(pyro_ctx* ctx, int steps, int batch, float lr, double* mean_loss);
/* Host-buffer test paths: network outputs for n feature rows, and the
 * gradient (6288 values) and loss sum of the negative log-likelihood. */
int pyro_tet_forward(pyro_ctx* ctx, const float* features, int n, float* out16);
/* The same on device buffers, stream-ordered, no allocation after the first
 * tcgen05 call (which allocates a 4-byte error flag). */
int pyro_tet_forward_device(pyro_ctx* ctx, const float* dev_features, int n, float* dev_out16);
/* Kernel of the batched forward: 1 (default) the 5th-generation tensor cores
 * (tcgen05.mma, accumulators in tensor memory, 128 rows per CTA), 0 the
 * mma.sync m16n8k16 kernel of the move and the training. A tcgen05 wait that
 * runs out returns PYRO_ERR_TIMEOUT. */
int pyro_tet_set_forward(pyro_ctx* ctx, int tensor_memory);
int pyro_tet_gradient(pyro_ctx* ctx, const float* features, const float* targets, int n,
                      float* grad, double* loss_sum);
/* Diagnostics of the learned move: one pass over the up-tetrahedra of FCC
 * corner `corner` of every replica of J1-only system `system`, with the
 * single-lane form (form 0, network on mma.sync) or the tcgen05 form
 * (form 3), at the learned-move counter's current value (the counter is not
 * advanced). The pass updates the spins like any other and writes, per
 * tetrahedron (record index rep * L^3 + cell), 56 floats to `records`: the
 * four spins before the move (12), their external fields (12), the network
 * outputs (16), the proposal (12), the log of the Metropolis-Hastings ratio
 * as evaluated, the decision (0 or 1), the test uniform and beta. A test
 * compares them with an FP64 restatement of the move. Synchronous. */
int pyro_tet_trace_pass(pyro_ctx* ctx, int system, int corner, int form, float* records);
/* Cycles with learned moves: n_metro Metropolis + n_or over-relaxation
 * sweeps, n_tet tetrahedron sweeps, energies and (if do_swap) an exchange,
 * replayed from a CUDA graph. */
int pyro_cycle_tet(pyro_ctx* ctx, int n_metro, int n_or, int n_tet, int do_swap, int n_cycles);

/* Energy and magnetisation without any device allocation.
 *
 * This entry point has no counterpart in the reference. It is for callers
 * that cannot call cudaMalloc: code that runs inside a memory pool or arena
 * which owns all device memory, a framework that forbids allocation once its
 * buffers are sized, or a process that cannot afford the allocations a
 * pyro_ctx makes. It needs no context. The caller passes the spins of
 * n_replicas replicas of one L lattice (the float4 layout above, device
 * memory, 16-byte aligned) and receives the FP64 energy per replica in
 * dev_energy[n_replicas] and, if dev_magnetisation3 is not NULL, the
 * magnetisation in dev_magnetisation3[3 * n_replicas] (both 8-byte aligned;
 * a misaligned pointer returns PYRO_ERR_ARG and launches nothing). The
 * energy is that of the isotropic Heisenberg model with the four couplings
 * J1, J2, J3 (through a site) and J3b (across a hexagon) only: it has no
 * field and no bond matrices, so for a context built with either it differs
 * from pyro_observables_device.
 *
 * Its working space is a fixed array inside the library of
 * PYRO_NOALLOC_MAX_PARTIALS partial sums (32 B each, 2 MiB), present on every
 * GPU that loads the library until the process exits. One partial covers
 * 2048 sites, so a call handles at most 16 L^3 n_replicas <=
 * 2048 * PYRO_NOALLOC_MAX_PARTIALS sites (e.g. 256 replicas at L = 32, 32 at
 * L = 64); larger requests return PYRO_ERR_ARG with a message on stderr and
 * launch nothing. The call runs on the current CUDA device, on `cuda_stream`
 * (NULL = default stream), and returns without waiting. The first call on
 * each device looks up the array's device address; make that first call
 * before any stream capture. That address is kept per device ordinal, so
 * only the device's primary context (the one the CUDA runtime uses) is
 * supported. All calls share the one array, so calls that
 * overlap on the GPU (other streams, other threads) race with each other:
 * order them on one stream. */
#define PYRO_NOALLOC_MAX_PARTIALS 65536
int pyro_observables_noalloc(const float* dev_spins_xyzw, int L, int n_replicas, double J1,
                             double J2, double J3, double J3b, double* dev_energy,
                             double* dev_magnetisation3, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* PYRO_H */
