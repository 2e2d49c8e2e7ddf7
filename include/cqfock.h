/*
 * cqfock.h -- C ABI of the B200 direct two-electron (J/K) Fock build.
 *
 * This is the drop-in boundary for ChronusQ's direct contraction path.  A thin
 * C++ shim (chronusq_public_b200/shim/cqf_chronusq_shim.hpp) keeps ChronusQ's
 * class signatures and calls these functions; integer status codes cross the
 * boundary, never exceptions.
 *
 * Reference interfaces replaced (paths within xsligroup/chronusq_public):
 *   cqf_basis_create      BasisSet::update + ShellPairData::computeShellPairs
 *                         (src/basisset/basisset.cxx:98-191, :652-706) and
 *                         DirectTPI::computeSchwarz
 *                         (src/particleintegrals/aointegrals/aointegrals_utilities.cxx:53-162),
 *                         cached per geometry as DirectTPI does
 *                         (include/particleintegrals/twopints/gtodirecttpi.hpp:30-141)
 *   cqf_two_body_contract GTODirectTPIContraction<MatsT,double>::twoBodyContract
 *                         (include/particleintegrals/twopints/gtodirecttpi.hpp:199-206)
 *                         -> directScaffoldNew
 *                         (include/particleintegrals/contract/direct.hpp:1412-2123)
 *   cqf_contraction       TwoBodyContraction<T> {X, AX, HER, contType}
 *                         (include/particleintegrals/twopints.hpp:59-75)
 *   CQF_COULOMB/EXCHANGE  TWOBODY_CONTRACTION_TYPE (twopints.hpp:31-41)
 *
 * Matrices are column-major N x N with leading dimension N (direct.hpp:1868),
 * N = number of AO functions; complex matrices are interleaved (re, im)
 * doubles, i.e. std::complex<double>.  AX is accumulated (+=) as on the
 * reference's multi-threaded path (direct.hpp:2047-2058); callers zero it
 * first, as FockBuilder::formRawGDInBatches does (fockbuilder/impl.hpp:131-137).
 */
#ifndef CQFOCK_H
#define CQFOCK_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CQF_OK = 0,
  CQF_EINVAL = 1,     /* bad argument (null pointer, size, unsupported l) */
  CQF_ENOMEM = 2,     /* device allocation failed */
  CQF_ECUDA = 3,      /* CUDA runtime error */
  CQF_ENOTSUP = 4,    /* feature not supported for these inputs */
  CQF_ETIMEDOUT = 5,  /* a bounded device/host wait ran out */
  CQF_ENODEV = 6      /* no CUDA device */
} cqf_status;

typedef enum { CQF_COULOMB = 0, CQF_EXCHANGE = 1 } cqf_contraction_type;

typedef enum { CQF_FP64 = 0, CQF_MIXED = 1 } cqf_precision;

/* One contracted shell, as libint2::Shell stores it in ChronusQ:
 * coeff are the libint-normalised contraction coefficients (contr[0].coeff),
 * pure = 1 for spherical (m = -l..l), 0 for Cartesian (x^l first). */
typedef struct {
  int l;
  int pure;
  int nprim;
  const double* alpha;
  const double* coeff;
  double origin[3]; /* Bohr */
} cqf_shell;

typedef struct cqf_basis cqf_basis;

/* One contraction: AX += G[X] (TwoBodyContraction<T>). */
typedef struct {
  const void* X;
  void* AX;
  int hermitian; /* TwoBodyContraction::HER */
  int type;      /* cqf_contraction_type */
} cqf_contraction;

typedef struct {
  int is_complex;       /* X/AX are std::complex<double> */
  int screen;           /* 1: Schwarz x density screen (reference default) */
  int device_pointers;  /* 1: X/AX are device pointers, 0: host pointers */
  int precision;        /* cqf_precision */
  double fp32_cutoff;   /* mixed: quartets with bound < cutoff run in FP32 */
  void* stream;         /* cudaStream_t to run on; NULL = the basis' stream */
  /* Work split over processes (the reference's MPI split of the shell-pair
   * loop, direct.hpp:1600-1604, 4C direct4C_libcint.hpp:933-936): with
   * shard_count > 1 a call computes only the quartets whose bra shell pair
   * (number p in the library's pair order) has p % shard_count ==
   * shard_index; the shards' results sum to the whole contraction (or 4C
   * build), and the caller sums them (the reference's MPIReduce,
   * direct.hpp:2085-2107).  AX is accumulated into, so give a prior value on
   * one shard only.  Defaults 0 / 1. */
  int shard_index;
  int shard_count;
} cqf_opts;

typedef struct {
  long long quartets_total;     /* unique quartets visited (8-fold) */
  long long quartets_screened;  /* dropped by the Schwarz x density screen */
  long long quartets_fp32;      /* computed on the FP32 path */
  long long quartets_fp64;      /* computed on the FP64 path */
  double device_ms;             /* device time of the contraction */
} cqf_stats;

/* Fill opts with the reference defaults (screen on, FP64, host pointers). */
void cqf_opts_default(cqf_opts* opts);

/* Upload shells, build significant shell pairs, primitive-pair data, class
 * buckets and Schwarz bounds on `device`.  thresh_schwarz is
 * DirectTPI::threshSchwarz_ (1e-12 in ChronusQ). */
cqf_status cqf_basis_create(const cqf_shell* shells, int nshell, double thresh_schwarz,
                            int device, cqf_basis** out);
cqf_status cqf_basis_destroy(cqf_basis* basis);

/* nbasis (AO functions), nshell, npair (significant shell pairs). */
cqf_status cqf_basis_info(const cqf_basis* basis, int* nbasis, int* nshell, int* npair);

/* Schwarz table, nshell x nshell column-major (host memory). */
cqf_status cqf_basis_schwarz(const cqf_basis* basis, double* Q);

/* Overlap S and kinetic T matrices (N x N column-major, host memory) of the
 * basis, computed on the device.  Replaces the one-electron overlap / kinetic
 * integrals ChronusQ takes from libint (used here to orthonormalise densities
 * and for the four-component metric). */
cqf_status cqf_basis_one_electron(cqf_basis* basis, double* S, double* T);

/* Nuclear-attraction matrix V (N x N column-major, host memory) of the basis
 * in the field of natom nuclei, nuclei[5 i .. 5 i + 4] = {Z, x, y, z (Bohr),
 * zeta}: zeta = 0 is a point charge (the libint2::Operator::nuclear engine
 * with charges -Z at the atoms, src/particleintegrals/aointegrals/
 * aointegrals_onee_drivers.cxx:139-145); zeta > 0 a Gaussian charge
 * Z (zeta/pi)^{3/2} exp(-zeta r^2) (finiteWidthNuc, the four-component
 * default; Molecule::computeCDist, src/molecule/molecule.cxx:197-226).
 * The reference's core Hamiltonian is T + V (stored as its scalar Pauli
 * component, 2 (T + V)); for four components its LL block is V. */
cqf_status cqf_basis_nuclear(cqf_basis* basis, int natom, const double* nuclei, double* V);

/* Derivative nuclear-attraction matrices of the four-component core
 * Hamiltonian, nuclei as for cqf_basis_nuclear: W (4 consecutive N x N
 * column-major host matrices) = pV.p, (pV x p)_x, (pV x p)_y, (pV x p)_z,
 * with (pV x p)_k = <d_i a|V|d_j b> - <d_j a|V|d_i b>, (i, j, k) cyclic
 * (the scalar / SOX / SOY / SOZ components of OnePRelInts,
 * src/particleintegrals/spatialtospinor.cxx:205-230). */
cqf_status cqf_basis_nuclear_pvp(cqf_basis* basis, int natom, const double* nuclei, double* W);

/* FourComponent::compute4CCH (src/fourcomp/fourcomp.cxx:36-100): the
 * four-component core Hamiltonian [[V, T], [T, W / (4c^2) - T]] as the four
 * Pauli components (scalar, MX, MY, MZ) the reference stores, each a 2N x 2N
 * complex column-major host matrix (LL block first): scalar = 2 x the
 * spin-free blocks, MX/MY/MZ = 2i (pV x p)_k / (4c^2) in the SS block. */
cqf_status cqf_four_comp_core_hamiltonian(cqf_basis* basis, int natom, const double* nuclei,
                                          void* const* H);

/* GTODirectTPIContraction::twoBodyContract: for each entry, AX += G[X]. */
cqf_status cqf_two_body_contract(cqf_basis* basis, const cqf_contraction* list, int n,
                                 const cqf_opts* opts, cqf_stats* stats);

/* Launch-shape autotuner (no counterpart in the reference, whose CPU loop has
 * no launch shapes).  Times the contraction `list` (as cqf_two_body_contract
 * would run it; X is read, AX is not touched) with each candidate launch
 * shape of the persistent class-quartet kernels -- 2, 4, 8 or 16 resident
 * blocks per SM requested -- every class timed alone between CUDA events,
 * and keeps the fastest per class pair in the basis for its later
 * contractions.  Complex Hermitian densities are tuned on the real split
 * they run as; contractions that run only on the generic kernels (which
 * have no launch shapes) return CQF_OK without timing anything.  With
 * cache_path, choices are looked up first and new ones appended, one line
 * per (GPU name, real / complex-split, class pair, size bucket
 * log2(nBra nKet), precision); cached values other than 2, 4, 8, 16 are
 * ignored, and *from_cache = 1 when every class pair was found there.  On
 * failure the basis keeps the shapes it had.  It allocates scratch
 * (cudaMalloc) and synchronises the device while timing. */
cqf_status cqf_autotune(cqf_basis* basis, const cqf_contraction* list, int n,
                        const cqf_opts* opts, const char* cache_path, int* from_cache);

/* CUDA-graph form of cqf_two_body_contract for builds repeated on the same
 * device buffers (many densities per launch, RT-TDDFT steps, response
 * right-hand sides).  cqf_graph_create captures the whole contraction once
 * (device pointers only; X and AX are bound at creation, AX += G[X] on every
 * launch); cqf_graph_launch replays it on `stream` (NULL = the basis' stream)
 * without synchronising.  Batched form of FockBuilder::formRawGDInBatches'
 * many-density call (include/fockbuilder/impl.hpp:109-244), as used by
 * MOIntsTransformer (include/mointstransformer/tpi_ssfock.hpp:378-379). */
typedef struct cqf_graph cqf_graph;
cqf_status cqf_graph_create(cqf_basis* basis, const cqf_contraction* list, int n,
                            const cqf_opts* opts, cqf_graph** out);
cqf_status cqf_graph_launch(cqf_graph* graph, void* stream);
cqf_status cqf_graph_destroy(cqf_graph* graph);

/* Size of the fixed scratch array of cqf_two_body_contract_noalloc. */
#define CQF_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)

/* Same contraction as cqf_two_body_contract (the same HER normalisation and
 * kernels, complex Hermitian densities included), but it allocates no device
 * memory: its scratch is one fixed CQF_NOALLOC_SCRATCH_BYTES array compiled
 * into the library (held by every GPU that loads the library until exit).
 * No counterpart in the reference (ChronusQ takes scratch from its memory
 * manager); it is for callers that cannot call cudaMalloc during the call,
 * e.g. inside a framework that owns all device memory.  The basis must
 * already exist: cqf_basis_create, which allocates, also resolves the
 * array's device address on its device.  CUDA loads kernel code lazily on a
 * kernel's first launch; a caller that must see no device allocation at all
 * in these calls runs one contraction of the same kind beforehand (or sets
 * CUDA_MODULE_LOADING=EAGER).  Calls needing more scratch than the array
 * holds return CQF_EINVAL.  All calls share the array and it keeps the last
 * call's contents (each call clears what must start at zero); calls that
 * overlap on the GPU race on it and must be serialised. */
cqf_status cqf_two_body_contract_noalloc(cqf_basis* basis, const cqf_contraction* list, int n,
                                         const cqf_opts* opts, cqf_stats* stats);

/* ---------------------------------------------------------------------
 * Four-component Dirac-Coulomb(-Gaunt) contraction.
 *
 * The (X, AX) entries of one relativistic contraction, in the order of
 * DIRAC_PAULI_SPINOR_COMP (include/particleintegrals/contract/
 * direct4C_libcint.hpp:279-310): Coulomb LL (MS), exchange LL (MS, MX, MY,
 * MZ), Coulomb SS (4), exchange SS (4), exchange LS (4) -- 17 entries --
 * and, for GAUNT and GAUGE only, Coulomb LS (4), Coulomb SL (4), exchange
 * SL (4) -- 29 entries.  Every X and AX is an N x N complex (interleaved re, im)
 * column-major matrix, N = nbasis.
 * --------------------------------------------------------------------- */
typedef enum {
  CQF_CLLMS = 0, CQF_XLLMS, CQF_XLLMX, CQF_XLLMY, CQF_XLLMZ,
  CQF_CSSMS, CQF_CSSMX, CQF_CSSMY, CQF_CSSMZ,
  CQF_XSSMS, CQF_XSSMX, CQF_XSSMY, CQF_XSSMZ,
  CQF_XLSMS, CQF_XLSMX, CQF_XLSMY, CQF_XLSMZ,
  CQF_REL_NMAT,
  CQF_CLSMS = CQF_REL_NMAT, CQF_CLSMX, CQF_CLSMY, CQF_CLSMZ,
  CQF_CSLMS, CQF_CSLMX, CQF_CSLMY, CQF_CSLMZ,
  CQF_XSLMS, CQF_XSLMX, CQF_XSLMY, CQF_XSLMZ,
  CQF_REL_NMAT_GAUNT
} cqf_rel_comp;

/* TYPE of the 4C contraction (entry 0's contType in the reference). */
typedef enum {
  CQF_REL_BARE_COULOMB = 0, CQF_REL_LLSS = 1, CQF_REL_SSSS = 2, CQF_REL_GAUNT = 3,
  CQF_REL_GAUGE = 4
} cqf_rel_type;

/* GTODirectRelERIContraction::twoBodyContract (include/particleintegrals/
 * twopints/gtodirectreleri.hpp:75-94) -> directScaffoldLibcint
 * (direct4C_libcint.hpp:138-2832) for one contraction type: every non-NULL
 * AX is zeroed (:313-314), then
 *   BARE_COULOMB: AX[CLLMS] = J[Re X[CLLMS]], AX[XLLM*] = K[X[XLLM*]] (:514-790)
 *   LLSS: AX[CLLMS], AX[CSSM*] (Coulomb, order c^-2) and, with
 *         compute_exchange, AX[XLSM*] (:810-1441)
 *   SSSS: AX[CSSM*] and, with compute_exchange, AX[XSSM*] (:1841-2832).
 *   GAUNT (29 entries, :2833-3907): AX[CLSM*] (Coulomb, LS block, from the
 *         LS and SL densities X[CLSM*], X[CSLM*]) and, with
 *         compute_exchange, AX[XLLM*] (from the SS density X[XSSM*]),
 *         AX[XSSM*] (from the LL density X[XLLM*]) and AX[XLSM*] (from the
 *         SL density X[XSLM*]); always FP64.  AX[CSLM*] and AX[XSLM*] are
 *         neither read nor written (the reference's list points them at the
 *         CLSM* / XLSM* outputs; such aliasing is allowed).
 *   GAUGE (29 entries, :3908-5160): the same entries and sites with the
 *         gauge kernel -(alpha_1 . r12)(alpha_2 . r12) / r12^3 of the Breit
 *         interaction in place of Gaunt's -alpha_1 . alpha_2 / r12.
 * Entries a type does not read or write may be NULL; only the entries a
 * type writes are zeroed.  The densities must be
 * Hermitian, as the reference requires (:144-145).  opts->is_complex is
 * ignored (always complex); opts->device_pointers, opts->stream, opts->screen
 * apply, and opts->precision = CQF_MIXED runs the quartets whose screening
 * bound is below opts->fp32_cutoff in FP32 arithmetic (digestion and
 * accumulation stay FP64; the reference is FP64 throughout). */
cqf_status cqf_rel_two_body_contract(cqf_basis* basis, const void* const* X, void* const* AX,
                                     int type, int compute_exchange, const cqf_opts* opts,
                                     cqf_stats* stats);

/* Hamiltonian switches of the 4C two-electron build (the reference's
 * HamiltonianOptions: BareCoulomb, DiracCoulomb, DiracCoulombSSSS, Libcint,
 * Gaunt, Gauge) and the exchange scaling xHFX. */
typedef struct {
  int bare_coulomb, dirac_coulomb, dirac_coulomb_ssss, libcint;
  double xHFX;
  int gaunt, gauge;
} cqf_dc_opts;
/* Defaults of the reference: bare Coulomb, Dirac-Coulomb and SSSS on,
 * libcint on, Gaunt and Gauge off, xHFX = 1. */
void cqf_dc_opts_default(cqf_dc_opts* o);

/* FourCompFock::formGDDirect (include/fockbuilder/fourcompfock/impl.hpp:
 * 3752-4636): D[4] = Pauli components (scalar, MX, MY, MZ) of the
 * 2N x 2N complex 4C density (column-major, LL block first); G[4] receives
 * twoeH - xHFX K with the 2C^2 / -C^2 / 2C^4 / -C^4 weights of the LLSS and
 * SSSS terms, the Gaunt and Gauge terms' 2C'^2 (LS Coulomb) and -C'^2 (LL,
 * SS, LS exchange), C'^2 = C^2, or C^2 / 2 with the gauge term on (the
 * Breit interaction; impl.hpp:4228-4540), twoeH_LL = 2 J (libcint) or J,
 * and the SL blocks set to the conjugate transpose of the LS blocks.  opts as for
 * cqf_rel_two_body_contract (CQF_MIXED applies to every contraction type of
 * the build but Gaunt and Gauge, the bare-Coulomb one included). */
cqf_status cqf_four_comp_gd(cqf_basis* basis, const void* const* D, void* const* G,
                            const cqf_dc_opts* dc, const cqf_opts* opts, cqf_stats* stats);

/* ---------------------------------------------------------------------
 * Nuclear-gradient contraction.
 *
 * DirectGradContraction::gradTwoBodyContract (include/particleintegrals/
 * gradints.hpp:278-283) -> directScaffoldGrad (include/particleintegrals/
 * contract/direct.hpp:2198-2571): for each of the nMat Hermitian real
 * matrices list[m].X (COULOMB or EXCHANGE; list[m].AX is not used) and each
 * nuclear coordinate (atom, xyz), the J- or K-type contraction of
 * d(mu nu|la si)/dR_{atom,xyz}, added into AX[(3 atom + xyz) * nMat + m]
 * (3 natom nMat N x N arrays) as 1/2 (A + A^T).  shell_atom[s] is the atom
 * of shell s (ChronusQ's mapSh2Cen).  Every quartet of significant pairs is
 * computed (the reference does not screen here); FP64; at most 8 matrices;
 * complex and non-Hermitian X are not built (the reference stops on the
 * latter).  opts: device_pointers, stream, shard_index / shard_count. */
cqf_status cqf_grad_two_body_contract(cqf_basis* basis, const int* shell_atom, int natom,
                                      const cqf_contraction* list, int nMat, void* const* AX,
                                      const cqf_opts* opts, cqf_stats* stats);

/* ---------------------------------------------------------------------
 * Fock-build server: requests of any basis size arrive at any time and
 * share one GPU (continuous batching).  No counterpart in the reference
 * (ChronusQ runs one build at a time); each request is the closed-shell
 * build FockBuilder::formRawGDInBatches performs for one density
 * (include/fockbuilder/impl.hpp:109-244): G = 2 J[D] - xHFX K[D].
 *
 * The server admits the oldest waiting request (FIFO) when an execution
 * slot is free and its device-memory footprint (cqf_fock_footprint) fits in
 * the budget that the running requests and the cached bases leave, evicting
 * idle cached bases (least recently used) to make room; a request alone on
 * the GPU is always admitted.  Every admitted request runs on its own worker
 * thread and its basis' own stream, so the set-up and kernels of different
 * requests overlap on the device.  Bases of recent geometries stay resident
 * (cache_entries), so a repeated geometry (SCF iterations, RT steps) skips
 * set-up.  A request's result depends only on its own inputs: the kernels
 * and work split are the same alone and in a mix (only the order of
 * floating-point atomics differs).
 * --------------------------------------------------------------------- */
typedef struct cqf_server cqf_server;

typedef struct {
  int device;
  int slots;                       /* requests on the GPU at once */
  unsigned long long mem_budget;   /* bytes for running requests + cached bases */
  int cache_entries;               /* bases kept resident after their request */
} cqf_server_opts;
/* device 0, 8 slots, 8 GiB, 16 cached bases. */
void cqf_server_opts_default(cqf_server_opts* o);

typedef struct {
  const cqf_shell* shells;   /* copied at submission */
  int nshell;
  double thresh_schwarz;     /* 1e-12 in ChronusQ */
  const double* D;           /* N x N real symmetric density, host, copied at submission */
  double* G;                 /* out: N x N host buffer, written on completion */
  double xHFX;               /* exchange scaling (1 for Hartree-Fock) */
  int precision;             /* cqf_precision */
  double fp32_cutoff;
} cqf_fock_request;

/* Per-request timing (milliseconds from submission) and outcome. */
typedef struct {
  cqf_status status;
  double queue_ms;    /* submission -> admission */
  double setup_ms;    /* basis set-up (0 when cached) */
  double build_ms;    /* J/K build and G */
  double latency_ms;  /* submission -> completion */
} cqf_request_info;

typedef struct {
  long long submitted, completed, failed;
  int peak_inflight;               /* most requests on the GPU at once */
  double p50_ms, p99_ms, mean_ms;  /* latency over completed requests */
} cqf_server_stats;

/* Device bytes a request of this basis is charged for: shell-pair data
 * (upper bound: every pair significant, every pair with the largest
 * primitive count) plus the contraction workspace of one J and one K
 * (densities and accumulators, norms, and the class kernels' quartet masks
 * and word lists: 16 B per 32 quartets of a bra pair and a ket tile in each
 * of three launch streams' regions, at most 4 MiB each). */
unsigned long long cqf_fock_footprint(const cqf_shell* shells, int nshell);

cqf_status cqf_server_create(const cqf_server_opts* opts, cqf_server** out);
/* Queues a request; *id identifies it in cqf_server_wait.  Returns without
 * waiting; G must stay valid until the request completes. */
cqf_status cqf_server_submit(cqf_server* server, const cqf_fock_request* req, long long* id);
/* Waits for request id (timeout_s < 0: no limit); fills info when it is
 * done.  Returns the request's status (its error text becomes this thread's
 * cqf_last_error), or CQF_ETIMEDOUT if it has not completed in time.  A
 * completed request is forgotten once a wait has returned its outcome. */
cqf_status cqf_server_wait(cqf_server* server, long long id, double timeout_s,
                           cqf_request_info* info);
cqf_status cqf_server_get_stats(cqf_server* server, cqf_server_stats* stats);
/* Finishes every submitted request, then frees the server and its bases. */
cqf_status cqf_server_destroy(cqf_server* server);

/* Text of the last error on this thread ("" if none). */
const char* cqf_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* CQFOCK_H */
