/*
 * or_ecycle.h -- C-ABI of the B200 explicit element cycle.
 *
 * One handle replaces, for the element groups handed to it, the in-scope body
 * of one OpenRadioss RESOL cycle:
 *
 *   FORINTC / FORINT          engine/source/engine/resol.F:4012, :4096
 *     (CFORC3 BT shells  engine/source/elements/shell/coque/cforc3.F:82,
 *      SFORC3 1-pt hexas engine/source/elements/solid/solide/sforc3.F:125)
 *   ASSPAR4 skyline sum       engine/source/assembly/asspar4.F:160-175
 *   element dt min            engine/source/engine/resol.F:5853-5858, :6080, :6226
 *   ACCELE                    engine/source/assembly/accele.F:63-123
 *   BCS10 / BCS1V             engine/source/constraints/general/bcs/bcs10.F:30
 *   VELOCITY                  engine/source/assembly/velocity.F:56-84
 *   DEPLA                     engine/source/assembly/displacement.F:69-110
 *
 * The calling convention follows the reference's own C-ABI precedent
 * (engine/source/coupling/coupling_c_interface.h: opaque handle, int status,
 * create / configure / advance / destroy) so that the Fortran engine binds it
 * with ISO_C_BINDING exactly like coupling_adapter.F90:50-150.
 *
 * Conventions
 *  - Every function returns 0 on success and a positive OR_E_* code on error;
 *    or_ecycle_last_error() returns the message.  The library never exits.
 *  - Arrays are plain host pointers in the reference's Fortran layouts:
 *      X, D, V, VR     3 x numnod, node-major   (X(3,NUMNOD))
 *      IXS             11 x nel, 1-based node numbers in rows 2..9 (NIXS=11)
 *      IXC             7 x nel,  1-based node numbers in rows 2..5 (NIXC=7)
 *      SIG (solid)     nel x 6, component-major  SIG(I+NEL*(J-1))
 *      SIG (shell IP)  npt x 5 x nel:  [ip][component][element]
 *  - The library copies inputs to device memory on the add/set calls and owns
 *    the device mirrors; the caller keeps ownership of its host arrays.
 *  - A handle holds one or more independent "parts"; each part has its own
 *    nodes, element groups and time step (one part = one reference domain).
 *  - The handle is not thread-safe; call it from one host thread.
 */
#ifndef OR_ECYCLE_H
#define OR_ECYCLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define OR_OK               0
#define OR_E_ARG            1   /* bad argument (null pointer, size, index)      */
#define OR_E_CUDA           2   /* CUDA runtime error                            */
#define OR_E_STATE          3   /* call out of order (e.g. step before finalize) */
#define OR_E_NEGVOL         4   /* zero/negative volume (SCHKJABT3, MSGID 166)    */
#define OR_E_DTMIN          5   /* element time step <= DTMIN (MQVISCB/CDT3)     */
#define OR_E_NAN            6   /* NaN/Inf in nodal acceleration                 */
#define OR_E_TIMEOUT        7   /* a bounded wait expired: the host's wait for a
                                   step, or a grid barrier of the persistent cycle */
#define OR_E_UNSUPPORTED    8   /* option outside the implemented path           */
#define OR_E_NOMEM          9   /* device allocation failed                      */

/* precision forms */
#define OR_PREC_FP64        0   /* plain FP64 everywhere ("-prec=dp")                    */
#define OR_PREC_SPLIT       1   /* FP32 element/material math, FP64 X, D, volumes, energies */

/* material laws */
#define OR_LAW_ELASTIC      1   /* /MAT/ELAST        (m1law.F, sigeps01c.F)           */
#define OR_LAW_JOHNSON_COOK 2   /* /MAT/PLAS_JOHNS   (m2law.F, sigeps02c.F, m2cplr.F) */

typedef struct or_ecycle or_ecycle;

typedef struct {
  int    precision;     /* OR_PREC_FP64 or OR_PREC_SPLIT                             */
  int    device;        /* CUDA device ordinal                                       */
  double dtfac_solid;   /* DTFAC1(1), default 0.9 (lectur.F:405-425)                 */
  double dtfac_shell;   /* DTFAC1(3), default 0.9                                    */
  double dtmin_solid;   /* DTMIN1(1); element dt <= this is OR_E_DTMIN               */
  double dtmin_shell;   /* DTMIN1(3)                                                 */
  double dtmx;          /* DTMX, default 1e20 (freform.F:584)                        */
  double dt_growth;     /* growth cap factor of resol.F:6080; the reference
                           multiplies by the REAL literal 1.1, i.e. (double)1.1f     */
  int    graph;         /* 1: replay step() through a captured CUDA graph            */
  int    block_hex;     /* threads per block, hex kernel: 64, 128 or 256; 0 = chosen
                           at finalize from the element count (64 while the patches
                           at 64 fit one wave of resident CTAs, else 128); the Python
                           autotuner times all three                                 */
  int    block_shell;   /* threads per block, shell kernel, likewise                 */
  int    block_node;    /* reserved, 0: the node pass runs tiles of 128 nodes, in the
                           form (register budget) the wave count selects            */
  int    persistent;    /* 0: the persistent shell cycle where eligible; -1: never
                           (see or_ecycle_persistent_info)                          */
} or_ecycle_config;

/* PM(.,MAT) entries used on the path (hm_read_mat02_jc.F90, m1law.F, m2law.F) */
typedef struct {
  int    law;           /* OR_LAW_*                                     */
  double rho0;          /* PM(1)                                        */
  double young;         /* PM(20)                                       */
  double nu;            /* PM(21)                                       */
  double shear;         /* PM(22)  G                                    */
  double bulk;          /* PM(32)  C1 / BULK                            */
  double a11;           /* PM(24)  E/(1-nu^2)                           */
  double a12;           /* PM(25)  nu*A11                               */
  double ssp_shell;     /* PM(27)  sqrt(E/rho)                          */
  double jc_a;          /* uparam(1) CA  (LAW2)                         */
  double jc_b;          /* uparam(2) CB                                 */
  double jc_n;          /* uparam(3) CN                                 */
  double epsmax;        /* uparam(4) EPMX, 1e20 when unset              */
  double sigmax;        /* uparam(5) SIGMX, 1e20 when unset             */
} or_material;

/* /PROP/SOLID values on the path (hm_read_prop14.F:338-380) */
typedef struct {
  double qa;            /* GEO(14), default 1.1   */
  double qb;            /* GEO(15), default 0.05  */
  double qh;            /* GEO(13), default 0.1   */
  int    jcvt;          /* IGEO(16) = Iframe - 1: 0 global frame (Jaumann stress
                           rotation), 1 convected frame of SRCOOR3 (sforc3.F:505,
                           :798-816, :1603-1614)                                  */
  int    pad;
} or_solid_prop;

/* /PROP/SHELL values on the path (hm_read_prop01.F:141-317) */
typedef struct {
  double thk;           /* GEO(1) initial thickness (used where THKE is not given) */
  int    npt;           /* integration points through the thickness, 1..10        */
  int    ithk;          /* 1: element uses the current thickness (ITHK>0)         */
  int    ipla;          /* M2CPLR return: 0 radial (Iplas 2), 1 Newton with three
                           iterations (Iplas 1), 2 normal projection + radial
                           (Iplas 3); cgrtails.F:822-829 maps Iplas to IPLA        */
  int    ishfram;       /* local frame: 0 (default) or 2 (/SHFRA/V4, contrl.F:478-486;
                           cnvec3.F:82-106)                                        */
  double hm, hf, hr;    /* GEO(13..15) hourglass coefficients                     */
  double shf;           /* shear factor SHF (5/6 for ISH=0)                       */
  double pressure;      /* uniform /PLOAD-style pressure on the group, Pa (0=none)*/
  double dn;            /* GEO(17) numerical damping Dn: the V-shape hourglass
                           coefficient of one-point shells (mhvis3.F)             */
  int    ishell;        /* Ishell of /PROP/SHELL as the starter leaves it
                           (hm_read_prop01.F:141-315): 0 or 1 Q4 with CHVIS3 shape
                           vectors (engine IHBE 1), 2 Q4 with plain hourglass
                           vectors (IHBE 0), 3 Q4 with warping terms and CHSTI3
                           elasto-plastic hourglass (IHBE 2), 4 Q4 with warping
                           terms (IHBE 4).  With npt = 1, Ishell 0 and 2 become 1
                           (hm_read_prop01.F:246-250) and the hourglass forces are
                           MHVIS3's.  Ismstr 2 throughout.                        */
  int    pad;
} or_shell_prop;

/* time-step state of one part, in/out of or_ecycle_step (RESOL scalars) */
typedef struct {
  double tt;            /* TT      */
  double dt1;           /* DT1     */
  double dt2;           /* DT2     */
  double dt12;          /* DT12    */
  double dt2old;        /* DT2OLD  */
  int    ncycle;        /* NCYCLE  */
  int    ityptst;       /* ITYPTS  element type that set DT2 (1 solid, 3 shell) */
  int    neltst;        /* NELTS   0-based element index in its part            */
  int    pad;
} or_ecycle_time;

/* energies of one part, FP64 (ecrit.F:300-363, sbilan.F, cbilan.F, shvis3.F) */
typedef struct {
  double internal;      /* sum EINT*V0 (solids) + EINT(1)+EINT(2) (shells)  */
  double kinetic;       /* 1/2 m |V + DT1/2 A|^2                            */
  double kinetic_rot;   /* 1/2 I |VR + DT1/2 AR|^2                          */
  double hourglass;     /* cumulative EHOUR                                 */
  double plastic_work;  /* cumulative sum sigma_y * dpla * volume           */
  double external_work; /* cumulative WFEXT of the /CLOAD and /PLOAD loads
                           (force.F90: 1/2 (F(t-dt1)+F(t)).v * DT2 per
                           concentrated load, F . sum v * DT1 per segment)  */
} or_energies;

/* --- lifecycle ---------------------------------------------------------- */
/* replaces: coupling_adapter_create / configure (coupling_c_interface.h) */
int  or_ecycle_create(const or_ecycle_config* cfg, or_ecycle** out);
/* replaces: coupling_adapter_destroy */
int  or_ecycle_destroy(or_ecycle* h);
const char* or_ecycle_last_error(const or_ecycle* h);

/* --- model upload (hot-path inputs stay resident in HBM) ----------------- */
/* Adds a part; returns its index in *part.  Node arrays: X/V/VR (3,numnod),
   MS/IN (numnod) from the starter (smass3.F:79, cinmas.F), ICODT/ICODR (numnod)
   3-bit /BCS codes (bcs1.F:52-100; 4=x, 2=y, 1=z).  vr, in, icodr may be NULL. */
int  or_ecycle_add_part(or_ecycle* h, int numnod, const double* x, const double* v,
                        const double* vr, const double* ms, const double* in,
                        const int* icodt, const int* icodr, int* part);

/* Adds an 8-node 1-point hexa group (SFORC3, Isolid=1, Iframe=1, Ismstr=4).
   ixs: 11 x nel (NIXS); vol0: GBUF%VOL initial volumes (may be NULL: computed). */
int  or_ecycle_add_hex_group(or_ecycle* h, int part, int nel, const int* ixs,
                             const or_material* mat, const or_solid_prop* prop,
                             const double* vol0, int* group);

/* Adds a 4-node Belytschko-Tsay shell group (CFORC3, Ishell 1, Ismstr 2).
   ixc: 7 x nel (NIXC); thke: initial thickness per element (may be NULL). */
int  or_ecycle_add_shell_group(or_ecycle* h, int part, int nel, const int* ixc,
                               const or_material* mat, const or_shell_prop* prop,
                               const double* thke, int* group);

/* Per-element LAW2 yield stress A of a shell group (replaces uparam(1) per
   element; used by the sensitivity workload).  jc_a: nel values, Pa. */
int  or_ecycle_set_shell_yield(or_ecycle* h, int group, const double* jc_a);

/* Rigid velocity link of the engine's /VEL/TRA and /VEL/ROT cards (frelnk.F:75-101,
   RLINK10 rlink10.F:60-90, RLINK1 rlink1.F): after ACCELE and BCS10, every node of
   the link takes the mass-weighted mean acceleration of the link's nodes in the
   directions of ic (4=x, 2=y, 1=z; weights MS) and the inertia-weighted mean
   rotational acceleration in the directions of icr (weights IN); BCS10 is then
   applied again (resol.F:7022, :7053, :7458).  nodes: nnod 1-based node numbers
   of the part; a node belongs to one link at most; global axes only (no skew).
   Before finalize; returns the link's index in *link. */
int  or_ecycle_add_rlink(or_ecycle* h, int part, int nnod, const int* nodes,
                         int ic, int icr, int* link);
/* Rigid body of /RBODY (RBYFOR rbyfor.F / RGBODFP rgbodfp.F at resol.F:5452,
   RBYVIT rbyvit.F / RGBODV rgbodv.F at resol.F:7515, kinetic energy as RBYCOR /
   RGBCOR rgbcor.F corrects it), after the starter's initialisation (INIRBY,
   inirby.F): the part's arrays given to or_ecycle_add_part already hold the main
   node at the body's centre of mass with the body's mass (MS) and its smallest
   principal inertia (IN); rby12 = the principal axes e1, e2, e3 (3 doubles each,
   RBY(1:9)) and the principal inertias (RBY(10:12)).  Each cycle the secondary
   nodes' forces and moments about the main node go to the main node, the
   principal frame turns with the body, Euler's equations give its rotational
   acceleration, and the secondary nodes follow the body's rigid motion.
   master: 1-based node number; slaves: nsl >= 3 distinct 1-based node numbers;
   a node belongs to one body at most and to no rigid link; no rotational BCS on
   the main node; no sensor, skew or surface.  Before finalize; returns the
   body's index in *body. */
int  or_ecycle_add_rbody(or_ecycle* h, int part, int master, int nsl, const int* slaves, const double* rby12,
                         int* body);
/* Changes the directions of a link between steps (an engine file that no longer
   lists it: ic = icr = 0). */
int  or_ecycle_set_rlink(or_ecycle* h, int link, int ic, int icr);

/* --- loads and skewed boundary conditions (FORCE, force.F90; BCS1V) -------- */
/* Time function of /FUNCT: npts points (x strictly ascending, npts >= 1),
   piecewise linear with linear extrapolation beyond both ends, one point =
   constant (FINTER, tools/curve/finter.F).  Returns its index in *func. */
int  or_ecycle_add_function(or_ecycle* h, int npts, const double* x, const double* y, int* func);

/* Concentrated loads of /CLOAD (force.F90, Parith/ON branch): on each of the nnod
   nodes (1-based), along direction dir (1..3 force x, y, z; 4..6 moment xx, yy,
   zz) of the global axes (skew = -1) or of skew frame `skew`, the value
   fscale * f(TT / ascale_x) at the time TT of the cycle's start.  Each node gets
   its own assembly slot, summed after the element contributions.  Abscissa time
   only (Itypfun 1), no sensor.  Before finalize. */
int  or_ecycle_add_cload(or_ecycle* h, int part, int nnod, const int* nodes, int dir, int skew,
                         int func, double ascale_x, double fscale, int* load);

/* Pressure loads of /PLOAD (force.F90, segment branch): seg holds 4 x nseg 1-based
   node numbers (n4 = 0 for a triangle).  A quadrangle adds
   p (x3 - x1) x (x4 - x2) / 8 to each of its four nodes, a triangle
   p (x3 - x1) x (x3 - x2) / 6 to each of its three, p = fscale * f(TT / ascale_x),
   with the coordinates at the cycle's start.  Before finalize. */
int  or_ecycle_add_pload(or_ecycle* h, int part, int nseg, const int* seg, int func,
                         double ascale_x, double fscale, int* load);

/* Fixed skew frame (/SKEW/FIX after the starter's orthonormalisation): axes9 =
   x', y', z' unit vectors, 3 doubles each (SKEW(1:9,ISK)).  Returns its index. */
int  or_ecycle_add_skew(or_ecycle* h, const double* axes9, int* skew);

/* Skew frame of each node's /BCS codes (numnod ints, -1 = global axes): the
   fixed directions are those of the frame (BCS1V, bcs1.F), for translations and
   rotations alike.  Before finalize. */
int  or_ecycle_set_bcs_skew(or_ecycle* h, int part, const int* skew);

/* Builds the Parith/ON assembly tables (element_pon_: ADSKY/IADS/IADC) on the
   device and allocates work buffers.  Must follow the last add_* call. */
int  or_ecycle_finalize(or_ecycle* h);

/* Restores nodes, element state and energy accumulators to the values given at
   upload (the state after finalize), keeping the device layout; used to replay
   a run (benchmarks, finite-difference sensitivity checks). */
int  or_ecycle_reset(or_ecycle* h);

/* --- the cycle ------------------------------------------------------------ */
/* Runs ncycles explicit cycles for every part.  t: one or_ecycle_time per part,
   read on entry and written on return.  Synchronous, bounded wait. */
int  or_ecycle_step(or_ecycle* h, int ncycles, or_ecycle_time* t);

/* --- download / upload for output and restart ---------------------------- */
/* One part's nodes in the caller's layout (3 doubles per node; any pointer may be
   NULL).  Synchronous; the host arrays are copied by DMA when they are pinned.
   The copies go through a device staging buffer of 3 doubles per node of the
   largest part, allocated by or_ecycle_finalize. */
int  or_ecycle_get_nodes(or_ecycle* h, int part, double* x, double* d,
                         double* v, double* vr);
int  or_ecycle_set_nodes(or_ecycle* h, int part, const double* x, const double* d,
                         const double* v, const double* vr);
/* solid state: sig (nel x 6 component-major), eint (per initial volume), rho,
   qvis, pla, epsd; any pointer may be NULL */
int  or_ecycle_get_hex_state(or_ecycle* h, int group, double* sig, double* eint,
                             double* rho, double* qvis, double* pla, double* epsd);
/* shell state: sig (npt x 5 x nel), pla (npt x nel), thk, hourg (3 x nel
   component-major), eint (2 x nel component-major); any pointer may be NULL */
int  or_ecycle_get_shell_state(or_ecycle* h, int group, double* sig, double* pla,
                               double* thk, double* hourg, double* eint);
/* Restart: element state in the layouts of the get_* calls (any pointer may be
   NULL: left as is), and the cumulative hourglass energy, plastic work and
   external work of a part before the restart (added to or_ecycle_energies).  With
   the nodes (or_ecycle_set_nodes) and the time state passed to or_ecycle_step,
   this resumes a run from the reference's restart file (RDRESB / WRRESTP).
   or_ecycle_reset returns to the state after finalize and clears the sums. */
int  or_ecycle_set_hex_state(or_ecycle* h, int group, const double* sig, const double* eint,
                             const double* rho, const double* qvis, const double* pla,
                             const double* epsd);
int  or_ecycle_set_shell_state(or_ecycle* h, int group, const double* sig, const double* pla,
                               const double* thk, const double* hourg, const double* eint);
int  or_ecycle_set_energy_sums(or_ecycle* h, int part, double hourglass, double plastic_work,
                               double external_work);
int  or_ecycle_energies(or_ecycle* h, int part, or_energies* e);

/* --- diagnostics ----------------------------------------------------------- */
/* Device error word of the last step: code (OR_E_*), element/node index. */
int  or_ecycle_error_info(or_ecycle* h, int* code, int* index);
/* Per-phase CUDA-event times of the last step, ms: [hex, shell, node, total]. */
int  or_ecycle_phase_times(or_ecycle* h, double* ms4);
/* Device time of one launch of each phase kernel, microseconds: [hex, shell,
   node] (0 for a phase without work).  Each kernel is launched `reps` times
   back to back from a CUDA graph, replayed between two events, on the state the
   last step left; the handle is then reset to its uploaded state, as by
   or_ecycle_reset.  For roofline measurement; no counterpart in the reference. */
int  or_ecycle_kernel_times(or_ecycle* h, int reps, double* us3);
/* Number of this library's kernel launches issued by the last step. */
int  or_ecycle_launch_count(or_ecycle* h, long long* n);
/* CUDA stream of the handle (cudaStream_t as void*), for event timing. */
int  or_ecycle_stream(or_ecycle* h, void** stream);
/* Bytes of device memory held by the handle. */
int  or_ecycle_device_bytes(or_ecycle* h, long long* bytes);
/* Whether or_ecycle_step runs the handle's cycles in the persistent form: one
   cooperative launch per call in which each CTA (one per SM) keeps its patches'
   element state in registers and their nodes in shared memory, with one grid
   barrier per cycle.  Chosen at finalize for one part of shell groups with no
   rigid links and no /CLOAD or /PLOAD loads, graph = 1, whose patches fit one
   wave; cfg.persistent = -1, or OR_ECYCLE_PERSISTENT=0 in the environment, turns
   it off.  It performs the per-phase kernels' operations in the same order, so
   its results are theirs bit for bit when floating-point contraction is off
   (the library built with -fmad=false); with FMA contraction the compiler may
   fuse a multiply-add in one kernel and not in the other, and the two agree to
   rounding.  ctas, threads: its launch shape (0 when off; either may be NULL).
   No counterpart in the reference. */
int  or_ecycle_persistent_info(or_ecycle* h, int* on, int* ctas, int* threads);

/* --- domain decomposition (one part split over ranks) ---------------------- */
/* The reference's SPMD cycle on one mesh: each rank runs a handle with its
   share of the elements and the nodes they touch (full nodal masses); per
   cycle, the ranks exchange the partial force/moment sums of the nodes they
   share (SPMD_EXCH_A, resol.F after FORINT) and take the minimum of their
   element time steps (SPMD_GLOB_MIN5).  The exchange itself is the caller's
   (NCCL over NVLink, or any transport):
     or_ecycle_spmd_begin(h, t)
     per cycle: or_ecycle_spmd_elements(h, my_buf)      element kernels + pack
                exchange (below) into bufs
                or_ecycle_spmd_nodes(h, bufs, nviews)    nodal phase
     or_ecycle_spmd_end(h, t)
   A buffer (or_ecycle_spmd_buffer_bytes bytes, device memory on the handle's
   device) holds nhalo force sums of 4 reals (x, y, z, unused), nhalo moment
   sums of 4 reals, then the 16-byte time-step reduction (two unsigned 64-bit
   keys, minimum wins); reals are double, or float for OR_PREC_SPLIT.
   spmd_elements packs this rank's partial sums at its halo slots.  bufs are
   nviews such buffers, one per rank in ascending rank order, all in this
   rank's slot numbering: this rank's own, and for other ranks their partial
   sums at the slots of the nodes they hold (zero elsewhere).  The node pass
   sets a halo node's force to the sum of the buffers' entries in that order,
   and takes the time step from the minimum of the buffers' reductions: the
   caller either passes every rank's buffer (an all-gather, nviews = ranks) or
   only its neighbours' with the all-rank minimum already in its own reduction
   (a neighbour exchange plus a 16-byte all-reduce, as the reference does).
   Either way every rank holding a node computes the same nodal update.  The
   per-cycle calls are asynchronous on the handle's stream, begin and end
   synchronous.
   or_ecycle_set_halo: the part's nodes shared with other ranks, as nloc
   (part-local node, halo slot in [0, nhalo)) pairs, the numbering of this
   rank's buffers; count_ke[i] = 0 when another rank counts the node's kinetic
   energy (NULL: all counted).
   One part per handle.  No counterpart in the reference's C interfaces: the
   reference does this exchange in Fortran over MPI. */
int  or_ecycle_set_halo(or_ecycle* h, int part, int nloc, const int* local_node, const int* halo_slot,
                        const int* count_ke, int nhalo);
int  or_ecycle_spmd_buffer_bytes(or_ecycle* h, long long* bytes);
int  or_ecycle_spmd_begin(or_ecycle* h, or_ecycle_time* t);
int  or_ecycle_spmd_elements(or_ecycle* h, void* dev_buf);
int  or_ecycle_spmd_nodes(or_ecycle* h, const void* dev_bufs, int nviews);
int  or_ecycle_spmd_end(or_ecycle* h, or_ecycle_time* t);

/* --- adjoint (design sensitivities) -------------------------------------- */
/* Response of or_ecycle_adjoint:
     J = w_disp * D(comp) of node `node` of part `part` after the call's cycles
       + w_plastic * plastic work accumulated by all shell elements over them. */
typedef struct {
  int    part;          /* part of the response node                                  */
  int    node;          /* 0-based node index within the part; < 0: no displacement   */
  int    comp;          /* 0 = x, 1 = y, 2 = z                                        */
  int    checkpoint;    /* cycles between state checkpoints (<= 0: 50)                */
  double w_disp;
  double w_plastic;
} or_adjoint_response;

/* Runs ncycles from the current state exactly like or_ecycle_step with the
   per-phase kernels (the handle ends in the same state, t is updated the same
   way; on a handle that steps with the persistent kernel the two agree to
   rounding, see or_ecycle_persistent_info), then the hand-written
   reverse of those cycles, and returns J and its gradient with respect to
   - dJ_dA:   the Johnson-Cook yield A of every shell element (shell groups in
              add order, elements in IXC order; 0 for LAW1 groups),
   - dJ_dthk: the thickness of every shell element at the start of the call
              (the THK state, and THKE where ITHK = 0 makes THKE the one used),
   - dJ_dms, dJ_din: the nodal masses and rotational inertias (parts in add
              order, nodes in part order), so that a caller whose masses depend
              on the thickness adds that chain itself.
   The time-step sequence of the forward run is held fixed: the gradient is
   exact when dt does not depend on the parameters, e.g. when DTMX is below
   every element time step.  The reverse recomputes each segment of
   r->checkpoint cycles from a stored state.  FP64 handles with shell groups
   only, global or skewed BCS, /CLOAD loads, no /PLOAD and no rigid links
   (OR_E_UNSUPPORTED otherwise).  Any output pointer may be NULL.
   No counterpart in the reference, which has no adjoint. */
int  or_ecycle_adjoint(or_ecycle* h, int ncycles, const or_adjoint_response* r, or_ecycle_time* t,
                       double* J, double* dJ_dA, double* dJ_dthk, double* dJ_dms, double* dJ_din);

/* --- entry point that allocates nothing ---------------------------------- */
/* No counterpart in the reference.  For callers that cannot let this library
   allocate device memory (for example an engine that reserves one device pool
   at start-up and must keep its footprint fixed through the time loop): runs
   ncycles of one FP64 hexa group (LAW1/LAW2) of one part on caller-owned
   device arrays, with the reference's own Parith/ON tables (iads: skyline slot
   of each of the 8 corners, adsky: node -> slot CSR, numnod+1 entries), and
   keeps its only scratch, the FSKY force skyline, in a static device array of
   OR_NOALLOC_MAX_SLOTS slots (8 MB, held by every GPU that loads the library).
   Larger groups are rejected with OR_E_ARG.  No cudaMalloc / cudaFree or other
   allocating call is made.
   The tables use the group's own slot numbering, 0-based: adsky[0] = 0,
   ascending, adsky[numnod] = 8*nel, and iads a permutation of 0..8*nel-1 that
   puts every corner among the slots of its own node (the engine's global
   LSKY numbering, shared with shells and other groups, must be renumbered).
   They are checked on the device before the first cycle; a table that fails
   returns OR_E_ARG with nothing written and the offending element (corner
   errors) or node (adsky errors) in t->neltst.  On a device error during the
   cycles (OR_E_NEGVOL, OR_E_NAN) t->neltst likewise holds the element or node.
   On success t->ityptst = 1 and t->neltst = the element that set the last DT2,
   as the handle path reports them.
   The first call on a device looks up the scratch address with that device
   current (under a lock, so first calls from several host threads are safe).
   The call is synchronous, with the bounded wait of or_ecycle_step
   (OR_ECYCLE_TIMEOUT_S, OR_E_TIMEOUT when it expires); it cannot be called
   inside a stream capture.  All calls share the scratch: calls that overlap on
   the GPU race.
   Arrays: x, d, v 3 x numnod; ms, icodt numnod; conn, iads 8 x nel (0-based);
   sig 6 x nel component-major; eint, rho, qvis, pla, epsd, vol0 nel.
   stream: a cudaStream_t (NULL = legacy default stream). */
#define OR_NOALLOC_MAX_SLOTS 262144
int  or_ecycle_hex_step_noalloc(int device, void* stream, int ncycles, or_ecycle_time* t,
                                int numnod, double* x, double* d, double* v, const double* ms,
                                const int* icodt, int nel, const int* conn, const int* iads,
                                const int* adsky, const or_material* mat, const or_solid_prop* prop,
                                double dtfac, double dtmx, double dt_growth, double* sig, double* eint,
                                double* rho, double* qvis, double* pla, double* epsd, const double* vol0);

#ifdef __cplusplus
}
#endif
#endif /* OR_ECYCLE_H */
