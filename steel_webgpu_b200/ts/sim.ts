// The reference's Sim (packages/steel-webgpu/src/sim.d.ts:53-92) over libsteel_b200.so through
// bun:ffi: a drop-in for code that steps scenes with `new Sim(device, scene, opts)`. SceneBuilder,
// loadScene and the URDF/MJCF loaders stay the reference's; the scene they produce (scene.json +
// scene.bin, sceneTypes.ts:91-99) goes to steel_scene_create, which packs it in C++ and steps it
// on one B200. There is no WebGPU device: the first constructor argument is the CUDA device
// ordinal (or a Context shared by several Sims).
//
// Bindings follow include/steel_b200.h; every call returns a status code and a failure throws
// Error(steel_last_error()), as the reference throws for unsupported scenes (sim.js:73, :128).
import { CString, dlopen, FFIType, ptr, type Pointer } from 'bun:ffi';

const LIB = process.env.STEEL_B200_LIB ?? new URL('../libsteel_b200.so', import.meta.url).pathname;

const { i32, u32, u64, f32 } = FFIType;
const P = FFIType.ptr;

export const symbols = {
  steel_last_error: { args: [], returns: FFIType.cstring },
  steel_ctx_create: { args: [i32, P], returns: i32 },
  steel_ctx_destroy: { args: [P], returns: i32 },
  steel_scene_create: { args: [P, P, u64, P, u64, P, P], returns: i32 },
  steel_batch_destroy: { args: [P], returns: i32 },
  steel_reset: { args: [P], returns: i32 },
  steel_step: { args: [P, u32], returns: i32 },
  steel_sync: { args: [P], returns: i32 },
  steel_step_timed: { args: [P, u32, P], returns: i32 },
  steel_scene_info_get: { args: [P, u32, P], returns: i32 },
  steel_read_poses: { args: [P, u32, P], returns: i32 },
  steel_newton_info: { args: [P, u32, P], returns: i32 },
  steel_state: { args: [P, u32, P, P, P, P], returns: i32 },
  steel_get_stats: { args: [P, u32, P], returns: i32 },
  steel_newton_dof: { args: [P, u32, u32, P], returns: i32 },
  steel_set_joint_target: { args: [P, u32, u32, f32, f32], returns: i32 },
  steel_set_joint_force: { args: [P, u32, u32, f32], returns: i32 },
  steel_set_body_wrench: { args: [P, u32, u32, P, P], returns: i32 },
  steel_set_body_pose: { args: [P, u32, u32, P, P], returns: i32 },
  steel_set_body_twist: { args: [P, u32, u32, P], returns: i32 },
  steel_copy_poses_device: { args: [P, u32, P, P], returns: i32 },
  steel_autotune: { args: [P, u32, P, P], returns: i32 },
  steel_set_team: { args: [P, u32], returns: i32 },
  steel_get_team: { args: [P, P], returns: i32 },
  steel_convex_hull: { args: [P, u32, P, P, P, P, P, P], returns: i32 },
} as const;

const lib = dlopen(LIB, symbols).symbols;

/** steel_set_team's default: a team launch for scenes of at least 2048 bodies or 64 articulations. */
export const TEAM_AUTO = 0xffffffff;

/** Convex hull of a point cloud as SceneBuilder.addConvexHull computes it (builder.js:61-173), in
 *  the library's C++ (steel_convex_hull): vertices, outward planes n . x = d and each face's
 *  vertices counter-clockwise about n. */
export function convexHull(points: Float64Array): { verts: Float64Array; planes: Float64Array; faces: number[][] } {
  const n = points.length / 3;
  const m = Math.max(n, 1);
  const verts = new Float64Array(3 * m);
  const planes = new Float64Array(8 * m);
  const start = new Uint32Array(2 * m + 1);
  const fv = new Uint32Array(6 * m);
  const counts = new Uint32Array(2);
  check(lib.steel_convex_hull(ptr(points), n, ptr(verts), ptr(planes), ptr(start), ptr(fv), ptr(counts),
                              ptr(counts.subarray(1))));
  const faces: number[][] = [];
  for (let k = 0; k < counts[1]; k++) faces.push(Array.from(fv.subarray(start[k], start[k + 1])));
  return { verts: verts.slice(0, 3 * counts[0]), planes: planes.slice(0, 4 * counts[1]), faces };
}

function check(rc: number): void {
  if (rc !== 0) throw new Error(`steel: ${String(lib.steel_last_error())}`);
}

/** One CUDA device and stream (the reference's GPUDevice role, device.js:7-26). */
export class Context {
  readonly handle: Pointer;
  constructor(readonly device = 0) {
    const out = new BigUint64Array(1);
    check(lib.steel_ctx_create(device, ptr(out)));
    this.handle = Number(out[0]) as Pointer;
  }
  destroy(): void {
    check(lib.steel_ctx_destroy(this.handle));
  }
}

export interface SimOptions {
  substeps?: number;
  iterations?: number;
  regularization?: number;
  warmStart?: number;
  colorWords?: number;
  solver?: Record<string, unknown>;
  /** Buffer capacities replacing the reference's fixed ones (MAXP, MAXC, MAXU, UH, WH, MAXDENSE, AH). */
  capacities?: Record<string, number>;
}

export interface SimStats {
  maxContacts: number;
  maxColors: number;
  maxUnits: number;
  maxPairs: number;
  contacts: number;
  colors: number;
  maxDense: number;
  asleep: number;
  overflow: string[];
  gpuFrameMs?: number;
}

export interface SimState {
  bodyQ: Float32Array;
  bodyQd: Float32Array;
  jointQ: Float32Array;
  jointQd: Float32Array;
}

/** The loaded scene the reference's loaders return: parsed scene.json plus scene.bin. */
export interface LoadedScene {
  json: { fps: number } & Record<string, unknown>;
  bin: ArrayBuffer;
}

const OVERFLOW = ['pairs', 'contacts', 'units', 'dense rows'];
const enc = new TextEncoder();

export class Sim {
  readonly scene: LoadedScene;
  readonly opts: SimOptions;
  readonly NB: number;
  readonly context: Context;
  readonly handle: Pointer;
  time = 0;
  frame = 0;
  private gpuFrameMs: number | undefined;
  private readonly ownsContext: boolean;

  constructor(device: number | Context, scene: LoadedScene, opts: SimOptions = {}) {
    this.ownsContext = typeof device === 'number';
    this.context = typeof device === 'number' ? new Context(device) : device;
    this.scene = scene;
    this.opts = opts;
    const json = enc.encode(JSON.stringify(scene.json));
    const bin = new Uint8Array(scene.bin);
    const o = enc.encode(JSON.stringify(opts) + '\0');
    const out = new BigUint64Array(1);
    check(lib.steel_scene_create(this.context.handle, ptr(json), json.length, ptr(bin), bin.length, ptr(o), ptr(out)));
    this.handle = Number(out[0]) as Pointer;
    const info = new Uint32Array(3);
    check(lib.steel_newton_info(this.handle, 0, ptr(info)));
    this.NB = info[0];
  }

  /** Like `new Sim`; the kernels are compiled ahead of time, so nothing runs off the main thread. */
  static async create(device: number | Context, scene: LoadedScene, opts?: SimOptions): Promise<Sim> {
    return new Sim(device, scene, opts);
  }

  destroy(): void {
    check(lib.steel_batch_destroy(this.handle));
    if (this.ownsContext) this.context.destroy();
  }

  reset(): void {
    check(lib.steel_reset(this.handle));
    this.time = 0;
    this.frame = 0;
  }

  /** Enqueues `frames` frames on the GPU; `timestamps` records their device time for stats(). */
  step(frames = 1, timestamps = false): void {
    if (timestamps) {
      const ms = new Float32Array(1);
      check(lib.steel_step_timed(this.handle, frames, ptr(ms)));
      this.gpuFrameMs = ms[0] / frames;
    } else {
      check(lib.steel_step(this.handle, frames));
    }
    this.frame += frames;
    this.time += frames / this.scene.json.fps;
  }

  /** `frames` frames, at most four in flight; onFrame(sim, frame) runs before each (sim.js:705-712). */
  async run(frames: number, onFrame?: (sim: Sim, frame: number) => unknown): Promise<void> {
    for (let i = 0; i < frames; i++) {
      if (onFrame) await onFrame(this, this.frame);
      this.step(1);
      if (i % 4 === 3) check(lib.steel_sync(this.handle));
    }
    check(lib.steel_sync(this.handle));
  }

  setJointTarget(newtonDof: number, pos: number, vel = 0): void {
    check(lib.steel_set_joint_target(this.handle, 0, this.portDof(newtonDof), pos, vel));
  }

  setJointTargets(pos: ArrayLike<number>, vel: ArrayLike<number> | null = null, first = 0): void {
    for (let k = 0; k < pos.length; k++) this.setJointTarget(first + k, pos[k], vel ? vel[k] : 0);
  }

  setJointForce(newtonDof: number, value: number): void {
    check(lib.steel_set_joint_force(this.handle, 0, this.portDof(newtonDof), value));
  }

  setBodyWrench(body: number, force: ArrayLike<number>, torque: ArrayLike<number>): void {
    check(lib.steel_set_body_wrench(this.handle, 0, body, ptr(Float32Array.from(force)), ptr(Float32Array.from(torque))));
  }

  setBodyPose(body: number, com: ArrayLike<number>, quat: ArrayLike<number>): void {
    check(lib.steel_set_body_pose(this.handle, 0, body, ptr(Float32Array.from(com)), ptr(Float32Array.from(quat))));
  }

  setBodyTwist(body: number, twist: ArrayLike<number>): void {
    check(lib.steel_set_body_twist(this.handle, 0, body, ptr(Float32Array.from(twist))));
  }

  /** Newton State (sim.js:732-763). */
  async state(): Promise<SimState> {
    const info = new Uint32Array(3);
    check(lib.steel_newton_info(this.handle, 0, ptr(info)));
    const s: SimState = {
      bodyQ: new Float32Array(info[0] * 7),
      bodyQd: new Float32Array(info[0] * 6),
      jointQ: new Float32Array(Math.max(info[1], 1)),
      jointQd: new Float32Array(Math.max(info[2], 1)),
    };
    check(lib.steel_state(this.handle, 0, ptr(s.bodyQ), ptr(s.bodyQd), ptr(s.jointQ), ptr(s.jointQd)));
    s.jointQ = s.jointQ.subarray(0, info[1]);
    s.jointQd = s.jointQd.subarray(0, info[2]);
    return s;
  }

  /** Per body: COM position (vec4) then quaternion x, y, z, w (vec4). */
  async poses(): Promise<Float32Array> {
    const out = new Float32Array(this.NB * 8);
    check(lib.steel_read_poses(this.handle, 0, ptr(out)));
    return out;
  }

  readPosesPooled(): Promise<Float32Array> {
    return this.poses();
  }

  /** The pose bridge (three/poseBridge.ts): poses GPU to GPU into a device buffer of NB BodyPose records. */
  copyPosesTo(devicePtr: Pointer, cudaStream: Pointer | null = null): void {
    check(lib.steel_copy_poses_device(this.handle, 0, devicePtr, cudaStream));
  }

  async stats(): Promise<SimStats> {
    const w = new Uint32Array(9);
    check(lib.steel_get_stats(this.handle, 0, ptr(w)));
    return {
      maxContacts: w[0],
      maxColors: w[1],
      maxUnits: w[2],
      maxPairs: w[3],
      contacts: w[4],
      colors: w[5],
      maxDense: w[6],
      asleep: w[7],
      overflow: OVERFLOW.filter((_, i) => (w[8] >> i) & 1),
      gpuFrameMs: this.gpuFrameMs,
    };
  }

  /** Picks the tile configuration for this scene (steel_autotune); resets the Sim. */
  autotune(frames = 3): {
    blockThreads: number;
    smemBudget: number;
    narrowBlocksPerSm: number;
    streamGroups: number;
    msPerFrame: number;
  } {
    const t = new Uint32Array(4);
    const ms = new Float32Array(1);
    check(lib.steel_autotune(this.handle, frames, ptr(t), ptr(ms)));
    this.time = 0;
    this.frame = 0;
    return { blockThreads: t[0], smemBudget: t[1], narrowBlocksPerSm: t[2], streamGroups: t[3], msPerFrame: ms[0] };
  }

  /** Blocks that prepare and solve this scene together (steel_set_team): 0 one block,
   *  TEAM_AUTO the default rule for large scenes, else that many. Returns the blocks in use. */
  setTeam(blocks: number = TEAM_AUTO): number {
    check(lib.steel_set_team(this.handle, blocks));
    const out = new Uint32Array(1);
    check(lib.steel_get_team(this.handle, ptr(out)));
    return out[0];
  }

  private portDof(newtonDof: number): number {
    const out = new Uint32Array(1);
    check(lib.steel_newton_dof(this.handle, 0, newtonDof, ptr(out)));
    return out[0];
  }
}

export { CString };
