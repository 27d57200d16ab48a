// cuda.ts — the reference app's solver interface on the B200 path (libwt.so through wt_napi.node).
//
// Drop-in for the WebGPU solver behind src/backend/types.ts: `SolverCUDA implements LbmSolver`
// (lines 7-16) and `cudaSolverFactory: SolverFactory` (line 18), plus the compute half of
// `Backend` (lines 24-53) as `CudaCompute`. Copy this file to src/backend/cuda.ts of the reference
// checkout and build the addon (binding.gyp beside this file); `CASES[c].run(cudaSolverFactory)`
// (src/analysis/validation.ts) then runs the reference's validation cases on the GPU unchanged.
import type { LbmSolver, SolverFactory } from './types';
import type { FieldExport, GridDims, SolverParams, SolverStats } from '../solver/types';
import type { MeshData, WheelDef } from '../voxelize/mesh';
import type { VoxelInfo } from '../voxelize/VoxelizerGPU';

// eslint-disable-next-line @typescript-eslint/no-var-requires
const wt = require('../../native/build/Release/wt_napi.node');

type Handle = unknown;

export class SolverCUDA implements LbmSolver {
  readonly n: number;
  stepCount = 0;
  private h: Handle | null;
  // calls on one handle must not overlap (the C ABI serialises nothing): chain them
  private chain: Promise<unknown> = Promise.resolve();

  constructor(readonly dims: GridDims, private p: SolverParams) {
    this.n = dims.nx * dims.ny * dims.nz;
    this.h = wt.create(dims, p);
  }

  uploadFlags(flags: Uint32Array): void {
    wt.uploadFlags(this.live(), flags);
  }

  uploadSdf(d: Float32Array): void {
    wt.uploadSdf(this.live(), d);
  }

  stepAndSample(steps: number): Promise<SolverStats> {
    const h = this.live();
    const run = this.chain.then(() => wt.stepAndSample(h, steps)) as Promise<SolverStats>;
    this.chain = run.catch(() => undefined);
    return run.then((s) => {
      this.stepCount = s.step;
      return s;
    });
  }

  setParams(p: Partial<SolverParams>): void {
    this.p = { ...this.p, ...p };
    wt.setParams(this.live(), this.p);
  }

  reset(): void {
    wt.reset(this.live());
  }

  clearStats(): void {
    wt.clearStats(this.live());
  }

  /** velocity texture of the last sample: (ux, uy, uz, rho) per cell */
  readVelocity(out: Float32Array = new Float32Array(4 * this.n)): Float32Array {
    wt.readVelocity(this.live(), out);
    return out;
  }

  destroy(): void {
    if (this.h) wt.destroy(this.h);
    this.h = null;
  }

  /** the native handle, for CudaCompute */
  handle(): Handle {
    return this.live();
  }

  private live(): Handle {
    if (!this.h) throw new Error('SolverCUDA: destroyed');
    return this.h;
  }
}

export const cudaSolverFactory: SolverFactory = (dims, p) => new SolverCUDA(dims, p);

/** The compute half of Backend (fits, createSolver, setParams, reset, clearStats, voxelize,
 *  exportFields, solverFactory); the renderer stays the reference's. */
export class CudaCompute {
  solver: SolverCUDA | null = null;

  fits(dims: GridDims, precision: 'f32' | 'f16' = 'f32'): boolean {
    return wt.fits(dims, { precision });
  }

  async createSolver(dims: GridDims, p: SolverParams): Promise<void> {
    this.solver?.destroy();
    this.solver = new SolverCUDA(dims, p);
  }

  setParams(p: Partial<SolverParams>): void {
    this.solver?.setParams(p);
  }

  reset(): void {
    this.solver?.reset();
  }

  clearStats(): void {
    this.solver?.clearStats();
  }

  async voxelize(mesh: MeshData | null, matrix: ArrayLike<number>, wheels: WheelDef[] = []): Promise<VoxelInfo> {
    const s = this.need();
    const w = new Float64Array(8 * wheels.length);
    wheels.forEach((d, k) => w.set([d.c[0], d.c[1], d.c[2], d.axis[0], d.axis[1], d.axis[2], d.r, d.hw], 8 * k));
    return wt.voxelize(s.handle(), mesh ? mesh.positions : null, mesh ? mesh.indices : null,
      Float64Array.from(matrix), w);
  }

  async exportFields(maxPoints: number): Promise<FieldExport> {
    return wt.exportFields(this.need().handle(), maxPoints);
  }

  solverFactory(): SolverFactory {
    return cudaSolverFactory;
  }

  private need(): SolverCUDA {
    if (!this.solver) throw new Error('CudaCompute: no solver');
    return this.solver;
  }
}
