/*
 * bgpu — B200-native rigid-body step, C ABI.
 *
 * Drop-in for the discrete-dynamics step of the Rust crates bullet-collision /
 * bullet-dynamics (CrazyboyQCD/bullet-physics). A world object owns all device
 * memory; caller buffers are borrowed for the duration of a call. One CUDA
 * stream per world; calls on one world are not thread-safe. Every call returns
 * a bgpu_status; bgpu_last_error() describes the last failure on the calling
 * thread.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   PhysicsWorld::new / with_broadphase      crates/bullet-dynamics/src/world.rs:406-463
 *   PhysicsWorld::set_gravity                crates/bullet-dynamics/src/world.rs:467-481
 *   PhysicsWorld::solver_info_mut            crates/bullet-dynamics/src/world.rs:956
 *   PhysicsWorld::add_body                   crates/bullet-dynamics/src/world.rs:524-563
 *   RigidBody::new_dynamic / new_static /    crates/bullet-dynamics/src/body.rs:388-499
 *     new_kinematic
 *   PhysicsWorld::step_simulation            crates/bullet-dynamics/src/world/step.rs:100-108
 *   PhysicsWorld::step_simulation_fixed      crates/bullet-dynamics/src/world/step.rs:136-199
 *   PhysicsWorld::body / body_mut            crates/bullet-dynamics/src/world.rs:566-598
 *   BroadPhase::compute_pairs_into           crates/bullet-collision/src/broadphase/mod.rs:94-130
 *   narrowphase::collide_seeded              crates/bullet-collision/src/narrowphase/mod.rs:63-286
 *   sequential_impulse::solve                crates/bullet-dynamics/src/solver/sequential_impulse.rs:692-705
 *   StepTimings                              crates/bullet-dynamics/src/timing.rs:20-117
 *   C-ABI handle pattern (demo_new/free/step) tools/wasm-demo/src/lib.rs:407-486
 */
#ifndef BGPU_H
#define BGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t bgpu_status;
#define BGPU_OK 0
#define BGPU_ERR_INVALID_ARGUMENT 1
#define BGPU_ERR_CAPACITY 2
#define BGPU_ERR_CUDA 3
#define BGPU_ERR_DEVICE_STATUS 4 /* a kernel left a bounded loop or overflowed a fixed buffer */
#define BGPU_ERR_NO_DEVICE 5

/* Bits of bgpu_step_stats.device_status (no counterpart in the reference, whose
 * step cannot fail: they report a bounded device loop or a fixed buffer that ran out). */
#define BGPU_DEVSTAT_UNION_FIND_LIMIT 0x002u  /* island union-find retries */
#define BGPU_DEVSTAT_BARRIER_TIMEOUT 0x004u   /* a grid barrier gave up waiting */
#define BGPU_DEVSTAT_COLOUR_OVERFLOW 0x008u   /* more than 128 PGS colours needed */
#define BGPU_DEVSTAT_EPA_CAPACITY 0x010u      /* EPA vertex/face budget */
#define BGPU_DEVSTAT_TRAVERSAL_STACK 0x040u   /* BVH traversal stack */
#define BGPU_DEVSTAT_COLOUR_ROUNDS 0x080u     /* colouring did not converge */
#define BGPU_DEVSTAT_MESH_CANDIDATES 0x100u   /* a convex-vs-mesh pair found over 64 candidate points */

/* Shape kinds (crates/bullet-collision/src/shapes/mod.rs:61-85, convex subset + plane). */
#define BGPU_SHAPE_SPHERE 0  /* params: radius */
#define BGPU_SHAPE_BOX 1     /* params: half extents x, y, z */
#define BGPU_SHAPE_CAPSULE 2 /* params: radius, half height (segment along local Y) */
#define BGPU_SHAPE_HULL 3    /* hull_points: n x 3 floats (must be convex) */
#define BGPU_SHAPE_PLANE 4   /* params: normal x, y, z, constant (static bodies only) */
#define BGPU_SHAPE_MESH 5    /* made by bgpu_add_mesh_shape / bgpu_add_heightfield_shape (static bodies only) */

/* Body flags (crates/bullet-dynamics/src/body.rs:204-252). */
#define BGPU_BODY_NO_CONTACT_RESPONSE 0x1u
#define BGPU_BODY_DISABLE_WORLD_GRAVITY 0x2u
#define BGPU_BODY_KINEMATIC 0x4u
#define BGPU_BODY_ADDITIONAL_DAMPING 0x10u

/* Activation states (crates/bullet-dynamics/src/body.rs:140-153). */
#define BGPU_ACTIVE 1u
#define BGPU_ISLAND_SLEEPING 2u
#define BGPU_WANTS_DEACTIVATION 3u
#define BGPU_DISABLE_DEACTIVATION 4u
#define BGPU_DISABLE_SIMULATION 5u

/* Contact subset of SolverInfo (crates/bullet-dynamics/src/solver/info.rs:24-107). */
typedef struct bgpu_solver_info {
    float erp2;                                /* 0.2 */
    float linear_slop;                         /* 0.005 */
    float restitution_velocity_threshold;      /* 1.0 */
    uint32_t split_impulse;                    /* 1 */
    float split_impulse_penetration_threshold; /* -0.04 */
    float split_impulse_turn_erp;              /* 0.1 */
    float warmstarting_factor;                 /* 0.85 */
    float global_cfm;                          /* 0.0 */
    float sor;                                 /* 1.0 */
    uint32_t num_iterations;                   /* 10 */
    float erp;                                 /* 0.2: joint position correction (info.rs erp) */
    float damping;                             /* 1.0: joint row velocity scale (info.rs damping) */
} bgpu_solver_info;

/* RigidBody construction parameters (body.rs:388-499). mass == 0 builds a static
 * body (new_static); the KINEMATIC flag builds new_kinematic. Zero sleeping
 * thresholds select the defaults 0.8 / 1.0; activation 0 selects the default. */
typedef struct bgpu_body_desc {
    uint32_t shape;
    float position[3];
    float orientation[4]; /* x, y, z, w */
    float linear_velocity[3];
    float angular_velocity[3];
    float mass;
    float friction;    /* default 0.5 */
    float restitution; /* default 0.0 */
    float linear_damping;
    float angular_damping;
    uint32_t flags;
    uint16_t group; /* default 1 */
    uint16_t mask;  /* default 0xFFFF */
    uint32_t activation;
    float linear_sleeping_threshold;
    float angular_sleeping_threshold;
} bgpu_body_desc;

/* Counters of the last step, and timing sums over the steps run since timing
 * was (re)enabled: the seven StepTimings stages (timing.rs:20-47), the PGS
 * kernel alone, and whole steps, all in ms of device time on the world's stream. */
typedef struct bgpu_step_stats {
    uint32_t num_bodies;
    uint32_t num_pairs;          /* broad-phase pairs */
    uint32_t num_contact_pairs;  /* pairs that emitted solver rows */
    uint32_t num_contacts;       /* solver rows */
    uint32_t num_colours;        /* PGS batches */
    uint32_t num_detect;         /* pairs that ran the narrow phase */
    uint32_t num_manifolds;      /* persistent manifolds after the step */
    uint32_t device_status;      /* or of the kernels' status bits (0 = clean) */
    uint32_t num_split_pairs;    /* row groups with split-impulse rows */
    uint32_t timed_steps;        /* steps in the sums below */
    float stage_ms[7];           /* integrate velocities, update aabbs, broadphase, islands,
                                    narrowphase, solve, integrate positions */
    float solve_kernel_ms;       /* the PGS kernel only (inside the solve stage) */
    float step_ms;
    uint32_t num_split_contacts; /* solver rows with an active split-impulse term */
} bgpu_step_stats;

/* Joints (constraint.rs:67-132: the point-to-point, fixed, hinge, gear, slider and cone-twist kinds). A frame is
 * the pivot followed by the basis columns x, y, z, in the body's centre-of-mass frame
 * (JointFrame, constraint.rs:658-682; the hinge axis is column z). Point-to-point joints
 * use only the frame origins (the pivots); gear joints (gear.rs) couple the spins about the
 * frames' z columns with gear_ratio; slider joints (slider.rs) slide along the frames' x
 * columns. Rows are rebuilt every step from the current
 * poses and solved after the contacts in each PGS sweep (sequential_impulse.rs:720-735);
 * a joint of a sleeping island (both bodies inactive) produces no rows. */
enum { BGPU_JOINT_POINT2POINT = 0, BGPU_JOINT_FIXED = 1, BGPU_JOINT_HINGE = 2, BGPU_JOINT_GEAR = 3, BGPU_JOINT_SLIDER = 4,
       BGPU_JOINT_SPRING2 = 5 /* added through bgpu_add_spring2_joints only */,
       BGPU_JOINT_CONETWIST = 6 /* ConeTwistConstraint, conetwist.rs: cone axis is the frames' x column */,
       BGPU_JOINT_GENERIC6DOF = 7 /* added through bgpu_add_generic6dof_joints only */ };
#define BGPU_JOINT_DISABLE_COLLISIONS 0x01u /* no contacts between the two bodies (default on) */
#define BGPU_JOINT_DISABLED 0x02u           /* set_enabled(false): no rows, no island link */
#define BGPU_JOINT_ANGULAR_ONLY 0x04u       /* hinge: skip the three pivot rows */
#define BGPU_JOINT_LIMIT 0x08u              /* hinge: angular limit [limit_low, limit_high] */
#define BGPU_JOINT_MOTOR 0x10u              /* hinge: motor (target velocity, max impulse) */
#define BGPU_JOINT_ERP 0x20u                /* point-to-point: own ERP instead of the solver's */
#define BGPU_JOINT_LIN_MOTOR 0x40u          /* slider: linear motor */
#define BGPU_JOINT_ANG_MOTOR 0x80u          /* slider: angular motor */
#define BGPU_JOINT_FRAME_B 0x100u           /* slider: linear reference frame B (use_linear_reference_frame_a off) */
#define BGPU_JOINT_CONE_MOTOR 0x200u        /* cone twist: motor toward cone_motor_target */
typedef struct bgpu_joint_desc {
    uint32_t kind;
    uint32_t body_a, body_b;
    uint32_t flags;
    float frame_a[12];
    float frame_b[12];
    float erp;           /* point-to-point, with BGPU_JOINT_ERP */
    float impulse_clamp; /* point-to-point: clamp of each row's impulse (0: none) */
    float limit_low, limit_high, limit_softness, limit_bias_factor, limit_relaxation; /* hinge */
    float motor_target_velocity, motor_max_impulse;                                    /* hinge */
    float gear_ratio;                                                                  /* gear */
    /* slider (SliderConstraint, slider.rs:8-60): limits (lower > upper frees the axis), */
    float lin_limit_low, lin_limit_high, ang_limit_low, ang_limit_high;
    /* softness / damping of the limits and of the orthogonal rows, */
    float softness_lim_lin, softness_lim_ang, damping_lim_lin, damping_lim_ang, softness_ortho_lin, softness_ortho_ang;
    /* motors (target velocity, max force) */
    float lin_motor_target_velocity, lin_motor_max_force, ang_motor_target_velocity, ang_motor_max_force;
    /* cone twist (conetwist.rs:86-135): swing spans about the frame's y and z axes and the twist
     * span about x (a span below 0.05 is a fixed or hinge configuration, a negative twist span
     * frees the twist), limit softness, bias and relaxation factors; */
    float swing_span1, swing_span2, twist_span, cone_softness, cone_bias_factor, cone_relaxation;
    /* the motor target in constraint space (x y z w, as set_motor_target_in_constraint_space stores
     * it) and its max impulse (negative: the swing row keeps its one-sided window) */
    float cone_motor_target[4];
    float cone_motor_max_impulse;
} bgpu_joint_desc;

/* Generic 6DOF spring-2 joints (Generic6DofSpring2Constraint, generic6dof_spring2.rs; Bullet's
 * btGeneric6DofSpring2Constraint). Axes 0-2 are linear along frame A's columns, 3-5 angular
 * about the relative-rotation axes of rotate_order (BGPU_ROTATE_*). Per axis: lower > upper
 * frees it, lower == upper locks it, lower < upper limits it with two one-sided elastic rows;
 * a motor (or position servo), and a damped spring toward equilibrium_point, may be added.
 * Axis fields mirror RotationalLimitMotor2 (:47-128) and TranslationalLimitMotor2 (:155-232).
 * stop_erp / stop_cfm / motor_erp / motor_cfm apply only with their BGPU_S2_* override flag
 * (setParam); without it the axis takes the solver's erp and global_cfm. Angular limits and
 * servo targets are taken as given (set_limit / set_servo_target normalise them on the
 * caller's side). */
enum { BGPU_ROTATE_XYZ = 0, BGPU_ROTATE_XZY = 1, BGPU_ROTATE_YXZ = 2, BGPU_ROTATE_YZX = 3, BGPU_ROTATE_ZXY = 4,
       BGPU_ROTATE_ZYX = 5 };
#define BGPU_S2_MOTOR 0x01u              /* enable_motor */
#define BGPU_S2_SERVO 0x02u              /* set_servo (with the motor) */
#define BGPU_S2_SPRING 0x04u             /* enable_spring */
#define BGPU_S2_STIFFNESS_LIMITED 0x08u  /* set_stiffness(.., limit_needed = true) */
#define BGPU_S2_DAMPING_LIMITED 0x10u    /* set_damping(.., limit_needed = true) */
#define BGPU_S2_STOP_ERP 0x20u           /* set_stop_erp override */
#define BGPU_S2_STOP_CFM 0x40u           /* set_stop_cfm override */
#define BGPU_S2_MOTOR_ERP 0x80u          /* set_motor_erp override */
#define BGPU_S2_MOTOR_CFM 0x100u         /* set_motor_cfm override */
typedef struct bgpu_spring2_axis {
    float lower_limit, upper_limit, bounce, stop_erp, stop_cfm, motor_erp, motor_cfm;
    float target_velocity, max_motor_force, servo_target, stiffness, damping, equilibrium_point;
    uint32_t flags; /* BGPU_S2_* */
} bgpu_spring2_axis;
typedef struct bgpu_spring2_desc {
    uint32_t body_a, body_b;
    uint32_t flags;        /* BGPU_JOINT_DISABLE_COLLISIONS, BGPU_JOINT_DISABLED */
    uint32_t rotate_order; /* BGPU_ROTATE_* */
    float frame_a[12];
    float frame_b[12];
    bgpu_spring2_axis axis[6];
} bgpu_spring2_desc;

typedef struct bgpu_world bgpu_world;

void bgpu_solver_info_default(bgpu_solver_info* out);
void bgpu_body_desc_default(bgpu_body_desc* out);
/* Cone twist: spans 1e30 (unlimited), softness 1, bias factor 0.3, relaxation 1, no motor
 * (identity target, max impulse -1).
 * Identity frames, collisions between the two bodies disabled, limit off (low 1 > high -1),
 * softness 0.9, bias factor 0.3, relaxation 1.0 (AngularLimit::new), gear ratio 1; slider:
 * linear axis free (1 > -1), rotation locked (0, 0), softness and damping 1 (SliderConstraint::new). */
void bgpu_joint_desc_default(bgpu_joint_desc* out);
/* Generic6DofSpring2Constraint::new: identity frames, collisions disabled, XYZ order, linear axes
 * locked at 0 (max motor force 0), angular axes free (1 > -1, max motor force 6); stop ERP 0.2,
 * motor ERP 0.9, everything else 0. */
void bgpu_spring2_desc_default(bgpu_spring2_desc* out);
/* Generic6DofSpring2Constraint::hinge2 (generic6dof_spring2.rs:329-377, Bullet's
 * btHinge2Constraint): the wheel joint from the two bodies' poses, a world anchor, the steering
 * axis axis1 and the spin axis axis2 (orthogonal): linear x/y locked, z a suspension spring
 * (stiffness 4 pi^2, damping 0.01, both auto-clamped) over [-1, 1], angular x free, y locked, z
 * limited to +-pi/4, equilibrium at the construction pose. Host arithmetic only. */
bgpu_status bgpu_spring2_hinge2(const float* pos_a, const float* quat_a, const float* pos_b, const float* quat_b,
                                const float* anchor, const float* axis1, const float* axis2, uint32_t body_a,
                                uint32_t body_b, bgpu_spring2_desc* out);

/* Library and device probes. */
const char* bgpu_version(void);
int bgpu_device_count(void);
size_t bgpu_last_error(char* buf, size_t len);
/* Makes `device` (0 .. bgpu_device_count() - 1, in the order this process sees the devices)
 * the calling thread's device for the library's later calls, as cudaSetDevice does for the
 * library's own CUDA runtime. A world lives on the device that was current when it was
 * created; use it from a thread with that device current. One process per GPU calls this
 * with its local rank before creating its worlds. */
bgpu_status bgpu_set_device(int device);

/* World lifetime (PhysicsWorld::new; world.rs:406-463). gravity may be NULL (0, -9.81, 0). */
bgpu_status bgpu_world_create(const bgpu_solver_info* info, const float* gravity, bgpu_world** out);
void bgpu_world_destroy(bgpu_world* w);
bgpu_status bgpu_world_set_gravity(bgpu_world* w, const float* gravity);
bgpu_status bgpu_world_set_solver_info(bgpu_world* w, const bgpu_solver_info* info);

/* Shapes and bodies (world.rs:524-563). */
bgpu_status bgpu_add_shape(bgpu_world* w, uint32_t type, const float* params, const float* hull_points,
                           uint32_t num_hull_points, uint32_t* out_shape);
/* Static triangle mesh (CollisionShape::triangle_mesh, shapes/triangle_mesh.rs:59-123):
 * nverts vertices (xyz) and ntris triangles (three vertex indices each). The library
 * builds the reference's BVH (shapes/bvh.rs:36-206) on the host. Meshes collide with
 * convex shapes (narrowphase/convex_mesh.rs:26-153) and take CCD sweeps
 * (convex_sweep.rs:305-345); a body with a mesh shape must be static. */
bgpu_status bgpu_add_mesh_shape(bgpu_world* w, const float* vertices, uint32_t nverts, const uint32_t* indices,
                                uint32_t ntris, uint32_t* out_id);
/* Heightfield (Heightfield::with_options, shapes/heightfield.rs:84-140), built into a
 * static triangle mesh: width x depth row-major heights, cell_size xyz (x and z used),
 * options: BGPU_HF_FLIP_QUAD_EDGES, BGPU_HF_DIAMOND, BGPU_HF_ZIGZAG, BGPU_HF_FLIP_WINDING,
 * and the up axis (BGPU_HF_UP_Y, the default, BGPU_HF_UP_X, BGPU_HF_UP_Z). */
#define BGPU_HF_FLIP_QUAD_EDGES 1u
#define BGPU_HF_DIAMOND 2u
#define BGPU_HF_ZIGZAG 4u
#define BGPU_HF_FLIP_WINDING 8u
#define BGPU_HF_UP_Y 0u
#define BGPU_HF_UP_X 16u
#define BGPU_HF_UP_Z 32u
bgpu_status bgpu_add_heightfield_shape(bgpu_world* w, const float* heights, uint32_t width, uint32_t depth,
                                       const float* cell_size, uint32_t options, uint32_t* out_id);
bgpu_status bgpu_add_bodies(bgpu_world* w, uint32_t n, const bgpu_body_desc* descs, uint32_t* out_first);
uint32_t bgpu_num_bodies(const bgpu_world* w);

/* Batched worlds (no counterpart in the reference, where every world is one
 * PhysicsWorld stepped on its own). A batch holds many independent worlds that
 * one sequence of kernel launches steps together: world k owns a contiguous
 * range of bodies, pairs only form inside a world (per-world all-pairs broad
 * phase), and each world keeps its own islands, sleeping and manifold-prune
 * state (step.rs:1006-1010 per world). Shapes are shared by all worlds. Every
 * other call (bgpu_step, bgpu_read_state, bgpu_apply_forces, ...) sees the batch
 * as one body array in world order. */
bgpu_status bgpu_batch_create(const bgpu_solver_info* info, const float* gravity, bgpu_world** out);
/* Appends n_worlds worlds whose bodies follow each other in descs (world k has
 * bodies_per_world[k] bodies); *out_first_world receives the first new world id. */
bgpu_status bgpu_batch_add_worlds(bgpu_world* w, uint32_t n_worlds, const uint32_t* bodies_per_world,
                                  const bgpu_body_desc* descs, uint32_t* out_first_world);
uint32_t bgpu_batch_num_worlds(const bgpu_world* w);
/* Writes num_worlds + 1 body offsets (world k owns bodies [offsets[k], offsets[k + 1])). */
bgpu_status bgpu_batch_world_offsets(bgpu_world* w, uint32_t* offsets);
/* Steps every world of the batch nsteps times (the same as bgpu_step). */
bgpu_status bgpu_batch_step(bgpu_world* w, float dt, uint32_t nsteps);

/* Launch shape of a batch's solver (no counterpart in the reference, which steps
 * one PhysicsWorld at a time: world/step.rs:100). Each world's PGS runs inside
 * one CTA, or one warp for worlds of at most warp_world_max_bodies bodies (the
 * world's row groups coloured and solved with the bodies' velocities in shared
 * memory, only block- or warp-local syncs between colour phases), with
 * threads_per_cta threads per CTA (32..256). threads_per_cta 0 selects the
 * global solver (one colouring and one cooperative PGS launch over all worlds).
 * A batch with joints, or a world too large for one CTA's shared memory, uses the
 * global solver. Either way each world equals its own sequential solve in the
 * order bgpu_read_solve_order reports. The launch shape must not change between
 * a tape's forward and backward passes. */
typedef struct bgpu_batch_tuning {
    uint32_t threads_per_cta;        /* 0: the global solver */
    uint32_t warp_world_max_bodies;  /* worlds with at most this many bodies: one per warp */
    uint32_t ctas;                   /* CTAs of the per-world launch (0: global solver in use) */
    uint32_t candidates;             /* configurations timed by the last bgpu_batch_autotune (0: none) */
    float ms_per_step;               /* the chosen configuration's device time per step then */
    float global_ms_per_step;        /* the global solver's device time per step in the same run */
} bgpu_batch_tuning;
/* Autotuner: from the batch's current state, times steps_per_candidate steps of
 * every candidate launch shape (threads per CTA 32 / 64 / 128 / 256 x warp-world
 * limits 0 / 32 / 64 / 128 / all, and the global solver), keeps the fastest, and
 * puts the batch back in the state it started from. out may be NULL. */
bgpu_status bgpu_batch_autotune(bgpu_world* w, float dt, uint32_t steps_per_candidate, bgpu_batch_tuning* out);
bgpu_status bgpu_batch_set_tuning(bgpu_world* w, uint32_t threads_per_cta, uint32_t warp_world_max_bodies);
bgpu_status bgpu_batch_get_tuning(bgpu_world* w, bgpu_batch_tuning* out);

/* Adjoint (no counterpart in the reference, whose world is not differentiable).
 * A tape steps its world forward, keeping a checkpoint of the world state every
 * checkpoint_every steps, then returns gradients of a loss of the final state with
 * respect to every body's initial linear and angular velocity, friction and
 * restitution. The differentiated model holds each step's contact geometry (rows,
 * world inverse inertia), its clamp decisions and its sleep decisions at their
 * forward values, and follows the warm start across steps (step.rs:751, 821); the
 * gyroscopic term is held fixed (it vanishes for isotropic inertia). The backward
 * pass replays each segment from its checkpoint, so its cost is about one extra
 * forward pass plus the reverse sweeps, and memory holds one segment's records.
 * The world must outlive the tape; bodies must not be added between forward and
 * backward. After backward the world is back in its state at the end of forward. */
typedef struct bgpu_tape bgpu_tape;
bgpu_status bgpu_tape_create(bgpu_world* w, uint32_t checkpoint_every, bgpu_tape** out);
void bgpu_tape_destroy(bgpu_tape* t);
/* Runs step_simulation(dt) nsteps times on the tape's world, recording checkpoints. */
bgpu_status bgpu_tape_forward(bgpu_tape* t, float dt, uint32_t nsteps);
/* grad_state: n x 9 floats per body, dL/d(position, linear velocity, angular velocity) of
 * the final state. Outputs (each may be NULL): grad_v0 and grad_w0 n x 3, grad_friction and
 * grad_restitution n (for the body's material coefficient; contacts combine them as products). */
bgpu_status bgpu_tape_backward(bgpu_tape* t, const float* grad_state, float* grad_v0, float* grad_w0,
                               float* grad_friction, float* grad_restitution);
/* Puts the world back in its state at the start of the last forward pass (body state and
 * manifold cache), e.g. to run the same rollout again after changing initial velocities. */
bgpu_status bgpu_tape_rewind(bgpu_tape* t);
/* Device time of the last forward and backward calls, in ms on the world's stream. */
bgpu_status bgpu_tape_timing(const bgpu_tape* t, float* forward_ms, float* backward_ms);

/* The step (step.rs:100-199). bgpu_step runs step_simulation(dt) nsteps times. */
bgpu_status bgpu_step(bgpu_world* w, float dt, uint32_t nsteps);
bgpu_status bgpu_step_simulation_fixed(bgpu_world* w, float dt, uint32_t max_sub_steps, float fixed_dt,
                                       uint32_t* out_substeps);
/* bgpu_step with device timing: *device_ms is the event-measured time on the
 * world's stream from before the first step to after the last one. */
bgpu_status bgpu_step_timed(bgpu_world* w, float dt, uint32_t nsteps, float* device_ms);

/* Body access (body / body_mut). State layout per body: pos3, quat4, linvel3,
 * angvel3, activation, deactivation time = 15 floats. Poses: pos3 + quat4. */
bgpu_status bgpu_read_state(bgpu_world* w, float* state);
bgpu_status bgpu_write_state(bgpu_world* w, const float* state);
bgpu_status bgpu_read_poses(bgpu_world* w, float* poses);
/* Accumulated force / torque per body (n x 3 each, either may be NULL);
 * cleared by the next step like RigidBody::clear_forces (step.rs:1272). */
bgpu_status bgpu_apply_forces(bgpu_world* w, const float* force, const float* torque);

/* Results of the last step, for inspection and parity checks.
 * Pairs: n x (lo, hi), lexicographic. Contacts: rows in solve order, 18 floats each:
 * body_a, body_b, point index, normal3, r_a3, r_b3, penetration, normal impulse,
 * tangent1 impulse, tangent2 impulse, push impulse, split flag.
 * Solve order: pair keys (lo << 32 | hi) in the order their rows were solved. */
bgpu_status bgpu_read_pairs(bgpu_world* w, uint32_t* pairs, uint64_t cap, uint64_t* out_n);
bgpu_status bgpu_read_contacts(bgpu_world* w, float* rows, uint64_t cap, uint64_t* out_n);
bgpu_status bgpu_read_solve_order(bgpu_world* w, uint64_t* keys, uint64_t cap, uint64_t* out_n);
/* PGS batches of the last step, one entry per colour in solve order: contact pairs
 * (row groups) in the batch, and those of them with split-impulse rows. Each solver
 * iteration runs one phase per colour, so these sizes set how the work spreads over
 * the device. Either array may be NULL; out_n receives the colour count. */
/* Joints (PhysicsWorld::add_constraint, world.rs): ids are consecutive from *first_id.
 * Rejects unknown kinds, out-of-range or equal bodies. */
bgpu_status bgpu_add_joints(bgpu_world* w, uint32_t n, const bgpu_joint_desc* d, uint32_t* first_id);
/* Continuous collision detection (RigidBody::ccd, body.rs:680-692) for bodies [first, first + n):
 * a dynamic, active body whose step motion |v dt| exceeds its motion threshold is swept as a
 * sphere of its swept-sphere radius against the other bodies of its world (those with contact
 * response, not joint-suppressed, passing group/mask, whose broad-phase box touches the swept
 * box) and its position is pulled back to the first hit after the integration
 * (step.rs:1068-1155, :1210-1214). A threshold or radius of 0 turns it off for that body. */
bgpu_status bgpu_set_ccd(bgpu_world* w, uint32_t first, uint32_t n, const float* motion_threshold,
                         const float* swept_sphere_radius);
/* Per body: the CCD clamp fraction of the last step (1 where no clamp happened). */
bgpu_status bgpu_read_ccd_clamps(bgpu_world* w, float* clamps);
/* Classic generic 6DOF joints (Constraint::generic_6dof, generic6dof.rs; Bullet's
 * btGeneric6DofConstraint), described by the spring-2 record, of which they read per axis the
 * limits (lower > upper free, else limited; angular ones normalised by the caller), the angular
 * bounce, stop_erp (always, no global fallback), and with BGPU_S2_MOTOR the motor's
 * target_velocity and max_motor_force; one limit-or-motor row per axis. Same id space as
 * bgpu_add_joints. bgpu_read_joint_spring2_state gives their Euler angles and pivot offset (with
 * fact_a 0.5 and has_static_body 0: this kind has no static-body split). */
bgpu_status bgpu_add_generic6dof_joints(bgpu_world* w, uint32_t n, const bgpu_spring2_desc* d, uint32_t* first_id);
/* Generic6DofConstraint::universal (generic6dof.rs:159-194, Bullet's btUniversalConstraint;
 * PhysicsWorld::add_universal): pivots at the world anchor, axis1 the frame z and axis2 the frame y
 * (orthogonal), linear and angular x locked, y within +-(pi/2 - 0.01), z within +-(pi - 0.01).
 * Host arithmetic only; add the result with bgpu_add_generic6dof_joints. */
bgpu_status bgpu_generic6dof_universal(const float* pos_a, const float* quat_a, const float* pos_b, const float* quat_b,
                                       const float* anchor, const float* axis1, const float* axis2, uint32_t body_a,
                                       uint32_t body_b, bgpu_spring2_desc* out);
/* Spring-2 joints (Constraint::generic_6dof_spring2), in the same id space as bgpu_add_joints. */
bgpu_status bgpu_add_spring2_joints(bgpu_world* w, uint32_t n, const bgpu_spring2_desc* d, uint32_t* first_id);
uint32_t bgpu_num_joints(bgpu_world* w);
/* Constraint::set_enabled / set_disable_collisions between steps (constraint.rs:637-652):
 * sets joint `id`'s BGPU_JOINT_DISABLE_COLLISIONS and BGPU_JOINT_DISABLED bits to `flags`
 * (any other bit is rejected); the next step uses them. Synchronises the world's stream. */
bgpu_status bgpu_set_joint_flags(bgpu_world* w, uint32_t id, uint32_t flags);
/* Per joint, 8 floats of the last step that built its rows (spring-2 joints; 0 for the other
 * kinds): the relative Euler angles (get_angle 0-2), the pivot offset in frame A
 * (get_relative_pivot_position 0-2), fact_a and has_static_body (0 or 1). */
bgpu_status bgpu_read_joint_spring2_state(bgpu_world* w, float* state);
/* Per joint: the hinge angle (HingeConstraint::hinge_angle) or the slider's angular position
 * (ang_pos) of the last step that built its rows; 0 for the other kinds. */
bgpu_status bgpu_read_joint_angles(bgpu_world* w, float* angles);
/* Per joint: the slider's linear position (SliderConstraint::lin_pos); 0 for the other kinds. */
bgpu_status bgpu_read_joint_positions(bgpu_world* w, float* positions);
/* Joint ids in the order their rows are solved (joint colour by colour). */
bgpu_status bgpu_read_joint_order(bgpu_world* w, uint32_t* ids, uint32_t cap, uint32_t* out_n);
/* Joint rows of the last step in solve order, 8 floats each: joint id, body_a, body_b,
 * effective mass, bias, limit kind, accumulated impulse, cfm. */
bgpu_status bgpu_read_joint_rows(bgpu_world* w, float* rows, uint32_t cap, uint32_t* out_n);
bgpu_status bgpu_read_colour_batches(bgpu_world* w, uint32_t* groups, uint32_t* split_groups, uint32_t cap,
                                     uint32_t* out_n);
bgpu_status bgpu_get_stats(bgpu_world* w, bgpu_step_stats* out);
/* Turns per-stage timing on (resetting the sums) or off. */
bgpu_status bgpu_enable_step_timing(bgpu_world* w, int on);
/* Diagnostics: runs one solver team barrier that nothing completes, with a time limit of
 * limit_ms (1..2000), and reports the device status bits it left (BGPU_DEVSTAT_BARRIER_TIMEOUT
 * when the wait gave up, as it must) and the device time the launch took. Shows that the
 * device-side waits of the step end with an error status instead of hanging the device. */
bgpu_status bgpu_selftest_wait_timeout(uint32_t limit_ms, uint32_t* device_status, float* waited_ms);

/* Stand-alone stages on caller data (parity harness entry points).
 * Broad phase: aabbs n x 6 (min3, max3) -> the closed-overlap pairs (i < j),
 * lexicographic; writes up to cap pairs and returns the count. */
bgpu_status bgpu_broadphase_pairs(const float* aabbs, uint32_t n, uint32_t* pairs, uint64_t cap, uint64_t* out_n);
/* Narrow phase on this world's shapes: per query shape_a/pose_a (pos3 quat4) vs
 * shape_b/pose_b; seeds n x 3 or NULL; out n x 4 x 7 (pos3, normal3, penetration),
 * counts n. force_convex != 0 routes every pair through GJK/EPA (convex_convex.rs:30). */
bgpu_status bgpu_collide(bgpu_world* w, uint32_t n, const uint32_t* shape_a, const float* pose_a,
                         const uint32_t* shape_b, const float* pose_b, const float* seeds, int force_convex,
                         float* out, uint32_t* counts);
/* Solver on this world's bodies: contacts n x 10 (body_a, body_b, pos3, normal3,
 * penetration, warm-start impulse); consecutive contacts of the same body pair form
 * one row group. Body velocities and push velocities are updated in place; the
 * rows (18 floats, as bgpu_read_contacts) come back in solve order, and the group
 * keys (body_a << 32 | body_b) in the order the groups were solved. */
bgpu_status bgpu_solve_contacts(bgpu_world* w, uint32_t n, const float* contacts, float inv_dt, float* rows_out,
                                uint64_t* order_keys_out);
/* Push velocities (n x 6: push_lin3, push_ang3) left by the last solve. */
bgpu_status bgpu_read_push(bgpu_world* w, float* push);

/* Broad phase that allocates nothing (no counterpart in the reference), for
 * callers that cannot allocate device memory while they run: loops with a fixed
 * device-memory budget, code inside a host runtime that owns the allocator, and
 * deadline-bound callers that cannot afford cudaMalloc / cudaFree (both may
 * synchronise the device). Same output as bgpu_broadphase_pairs, but the inputs
 * and outputs are device buffers: aabbs_dev n x 6 floats (min3, max3); pairs_dev
 * room for cap pairs of 2 x uint32, 8-byte aligned. *out_n receives the pair
 * count (also when it exceeds cap, which returns BGPU_ERR_CAPACITY). All scratch
 * lives in one fixed file-scope device array of the library (24 MiB on every GPU
 * that loads the library, held until exit), which limits n to
 * BGPU_NOALLOC_MAX_PROXIES and the unbounded proxies (extent >= 1e15, such as
 * planes) to BGPU_NOALLOC_MAX_UNBOUNDED; larger inputs return BGPU_ERR_CAPACITY.
 * The first call on a device looks up the array's device address: make it
 * before any stream capture. Every call shares the array, so calls that overlap
 * on the GPU race and must be serialised by the caller. stream is a
 * cudaStream_t (NULL = the default stream). Every call, not only the first,
 * copies the pair count to host memory and synchronises that stream before it
 * sizes the output, and it returns after its work on the stream has finished. */
#define BGPU_NOALLOC_MAX_PROXIES 65536u
#define BGPU_NOALLOC_MAX_UNBOUNDED 16u
bgpu_status bgpu_broadphase_pairs_noalloc(const float* aabbs_dev, uint32_t n, uint32_t* pairs_dev, uint64_t cap,
                                          uint64_t* out_n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BGPU_H */
