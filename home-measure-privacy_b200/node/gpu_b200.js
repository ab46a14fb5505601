// gpu_b200.js -- the reference trainer's GPU module (trainer/gpu.js of
// barakatiass-alt/home-measure-privacy) with its WebGPU work replaced by the B200
// library libgsb200.so, called through the Node-API addon gsb200_addon.cc.
//
// createRenderer() keeps the reference's surface (trainer/gpu.js:704-980, :979):
//   { device, render, gradients, train, trainScene, lossGradientOf }
// with the same arguments, Promises and thrown Errors, plus
//   forward(gaussians, cams) / backward(dLdImages)  -- the differentiable render as a
//     Function pair (what torch.autograd.Function is in Python): forward keeps the tile
//     lists and each pixel's final transmittance and last contributor on the device,
//     backward replays the blend in reverse from them,
//   destroy()  -- releases the device memory now instead of at garbage collection.
// Gaussians are the reference's objects {mean[3], logScale[3], rotation[4] (w, x, y, z),
// opacityLogit, color[3]}, optionally with `sh` (3 * ((shDegree + 1)^2 - 1) floats,
// channel-major like a .ply's f_rest_*); cameras are trainerCamera()'s
// {view[12], fx, fy, cx, cy, width, height} (trainer/colmap.js:57-64).
//
// Calls on one renderer run one after another (the library's context is not
// re-entrant); each resolves when its work is done, as the WebGPU read-backs do.
import { createRequire } from 'node:module';

const require = createRequire(import.meta.url);
const addon = require('./build/Release/gsb200.node');

/** Floats per Gaussian in the library's host record at an SH degree. */
export const paramStride = (degree) => 14 + 3 * ((degree + 1) ** 2 - 1);

/** Gaussian objects -> host records (n x paramStride(degree) floats). */
export function toRecords(gaussians, degree = 0) {
  const S = paramStride(degree);
  const nk = (degree + 1) ** 2 - 1;
  const out = new Float32Array(gaussians.length * S);
  gaussians.forEach((g, i) => {
    const o = i * S;
    out.set(g.mean, o);
    out.set(g.logScale, o + 3);
    out.set(g.rotation, o + 6);
    out[o + 10] = g.opacityLogit;
    out.set(g.color, o + 11);
    if (nk && g.sh) out.set(g.sh.slice(0, 3 * nk), o + 14);
  });
  return out;
}

/** Host records -> Gaussian objects (with `sh` above degree 0). */
export function fromRecords(data, degree = 0) {
  const S = paramStride(degree);
  const out = [];
  for (let o = 0; o + S <= data.length; o += S) {
    const g = {
      mean: [data[o], data[o + 1], data[o + 2]],
      logScale: [data[o + 3], data[o + 4], data[o + 5]],
      rotation: [data[o + 6], data[o + 7], data[o + 8], data[o + 9]],
      opacityLogit: data[o + 10],
      color: [data[o + 11], data[o + 12], data[o + 13]],
    };
    if (S > 14) g.sh = Array.from(data.subarray(o + 14, o + S));
    out.push(g);
  }
  return out;
}

/** packGaussians (trainer/gpu.js:688-694): the reference's 16-float GPU layout. */
export function packGaussians(gaussians) {
  const data = new Float32Array(gaussians.length * 16);
  gaussians.forEach((g, i) => {
    data.set([...g.mean, 0, ...g.logScale, g.opacityLogit, ...g.rotation, ...g.color, 0], i * 16);
  });
  return data;
}

/** unpackGaussians (trainer/gpu.js:602-609). */
export function unpackGaussians(data) {
  const out = [];
  for (let i = 0; i < data.length / 16; i++) {
    const d = data.subarray(i * 16, i * 16 + 16);
    out.push({ mean: [d[0], d[1], d[2]], logScale: [d[4], d[5], d[6]], opacityLogit: d[7], rotation: [d[8], d[9], d[10], d[11]], color: [d[12], d[13], d[14]] });
  }
  return out;
}

/** Indices 0..n-1 in a random order (Fisher-Yates), as trainScene's rounds take them. */
export function shuffled(n) {
  const order = Array.from({ length: n }, (_, i) => i);
  for (let i = n - 1; i > 0; i--) {
    const j = Math.floor(Math.random() * (i + 1));
    [order[i], order[j]] = [order[j], order[i]];
  }
  return order;
}

/** sceneExtent(views) (trainer/gpu.js:564-568), computed by the library. */
export function sceneExtent(views) {
  return addon.sceneExtent(views.map((v) => v.cam));
}

/**
 * createRenderer({gpuTiles}) (trainer/gpu.js:704-712).  `gpuTiles: false` keeps the
 * reference's CPU tileLists rectangle (the binning itself always runs on the GPU).
 * Extra options: shDegree (0..3), device (CUDA ordinal), near, batched, useGraph,
 * autotune, tileCull.  Throws Error when no CUDA device is visible (there is no CPU path).
 */
export async function createRenderer({ gpuTiles = true, shDegree = 0, device = 0, ...opts } = {}) {
  const ctx = addon.create({ gpuTiles, shDegree, device, ...opts });
  const degree = shDegree;
  let queue = Promise.resolve();
  // One call at a time on this context; a failed call rejects its own promise only.
  const serial = (fn) => {
    const p = queue.then(fn);
    queue = p.catch(() => {});
    return p;
  };
  const upload = (gaussians) => addon.setGaussians(ctx, toRecords(gaussians, degree), degree);
  const pixelsOf = (cams) => cams.reduce((a, c) => a + c.width * c.height, 0);

  /** Renders the Gaussians from one camera; RGB floats (width * height * 3). */
  const render = (gaussians, cam) =>
    serial(() => {
      upload(gaussians);
      return addon.render(ctx, cam);
    });

  /** gradients (trainer/gpu.js:826-839): {image, grads (n * 16), shape (n * 10)}. */
  const gradients = (gaussians, cam, target, ssim = 0) =>
    serial(() => {
      upload(gaussians);
      return addon.gradients(ctx, cam, Float32Array.from(target), ssim);
    });

  /** lossGradientOf (trainer/gpu.js:962-977): dLoss/dPixel, the reference's 7x7 SSIM. */
  const lossGradientOf = (image, target, width, height, lambda) =>
    serial(() => addon.lossGradient(ctx, Float32Array.from(image), Float32Array.from(target), width, height, lambda, 0));

  /** train (trainer/gpu.js:846-878): L1, one view per step in order, a loss per step. */
  const train = (gaussians, views, steps, lr = { color: 0.05, opacity: 0.05, mean: 0.002, scale: 0.01, rotation: 0.005 }) =>
    serial(async () => {
      upload(gaussians);
      addon.setViews(ctx, views.map((v) => v.cam));
      views.forEach((v, k) => addon.setTargetF32(ctx, k, Float32Array.from(v.target)));
      const losses = await addon.train(ctx, steps, lr);
      return { gaussians: fromRecords(await addon.getGaussians(ctx, degree), degree), losses: Array.from(losses) };
    });

  /**
   * trainScene (trainer/gpu.js:890-959): every photo once per round in a shuffled order,
   * one view per step; gradient statistics every step and densification on the device
   * every `densifyEvery` steps in [densifyFrom, densifyUntil] (split above 1 % of the
   * scene extent; with `prune`, drop above 10 %); the opacity reset halfway with
   * `opacityReset`; the step's loss sampled every 25 steps and reported through
   * `onProgress` every 50, which is awaited so the caller can pause.  Views hold
   * {cam, image: Uint8Array RGB}.  Returns the trained Gaussians.
   */
  const trainScene = (start, views, { steps = 3000, densifyEvery = 100, densifyFrom = 300, densifyUntil = 2000, maxSplats = 400000, ssim = 0, prune = false, opacityReset = false, onProgress, shouldStop, lr, seed = 0 } = {}) =>
    serial(async () => {
      lr = { color: 0.025, opacity: 0.05, mean: 0.002, scale: 0.005, rotation: 0.001, ...lr };
      upload(start);
      addon.setViews(ctx, views.map((v) => v.cam));
      views.forEach((v, k) => addon.setTargetU8(ctx, k, v.image));
      const extent = sceneExtent(views);
      const resetAt = opacityReset ? Math.round((densifyFrom + densifyUntil) / 2 / densifyEvery) * densifyEvery : -1;
      const lowOpacity = Math.log(0.01 / 0.99);
      addon.setDensifyStats(ctx, true);
      let order = [];
      let lossSum = 0, lossCount = 0;
      try {
        for (let t = 1; t <= steps; t++) {
          if (shouldStop?.()) break;
          if (!order.length) order = shuffled(views.length);
          const view = order.pop();
          const sample = t % 25 === 0;
          const loss = await addon.trainStep(ctx, lr, { ssim, window: 0 }, view, 1, sample);
          if (sample) {
            lossSum += loss;
            lossCount++;
          }
          if (t >= densifyFrom && t <= densifyUntil && t % densifyEvery === 0) {
            // The reference's threshold is per pixel of its first view (trainer/gpu.js:939-940).
            const gradThreshold = 2e-4 / (0.5 * views[0].cam.width);
            await addon.densify(ctx, { gradThreshold, maxCount: maxSplats, sizeThreshold: 0.01 * extent, maxSize: prune ? 0.1 * extent : Infinity, seed: seed * 1000003 + t });
            if (t === resetAt) addon.resetOpacity(ctx, lowOpacity);
          }
          if (t % 50 === 0) {
            await onProgress?.({ step: t, loss: lossCount ? lossSum / lossCount : NaN, count: addon.numGaussians(ctx) });
            lossSum = 0;
            lossCount = 0;
            await new Promise((r) => setTimeout(r));
          }
        }
        return fromRecords(await addon.getGaussians(ctx, degree), degree);
      } finally {
        addon.setDensifyStats(ctx, false);
      }
    });

  /**
   * The forward half of the Function pair: renders `cams` (all in one batched launch)
   * from `gaussians` and returns their images concatenated (HWC RGB floats per camera).
   * Keeps the tile lists, final transmittance and last contributor for backward().
   */
  const forward = (gaussians, cams) =>
    serial(() => {
      upload(gaussians);
      addon.setViews(ctx, cams);
      return addon.forward(ctx, 0, cams.length, pixelsOf(cams));
    });

  /**
   * The backward half: dLoss/dImages (same layout as forward's images; null = the
   * gradient of the last loss() against setTarget photos) back through the blend and the
   * projection.  Returns dLoss/dParameters as host records (n x paramStride(shDegree)).
   */
  const backward = (dLdImages) =>
    serial(() => addon.backward(ctx, dLdImages ? Float32Array.from(dLdImages) : null, degree));

  /** Loss of the last forward against per-view photos (setTarget), kept for backward(null). */
  const loss = (lambda = 0.2, window = 1) => serial(() => addon.loss(ctx, lambda, window));
  const setTarget = (view, image) =>
    serial(() => (image instanceof Uint8Array ? addon.setTargetU8(ctx, view, image) : addon.setTargetF32(ctx, view, Float32Array.from(image))));

  /** The context's Gaussians as objects. */
  const getGaussians = () => serial(async () => fromRecords(await addon.getGaussians(ctx, degree), degree));

  /** fromPly (trainer/gpu.js:983-999) into the context, f_rest bands up to shDegree; the count. */
  const loadPly = (bytes) => serial(() => addon.loadPly(ctx, new Uint8Array(bytes)));
  /** toPly (trainer/gpu.js:524-531) of the context's Gaussians (withSh adds f_rest_*): an ArrayBuffer. */
  const savePly = (withSh = false) => serial(() => addon.savePly(ctx, withSh));
  /** toSplat (trainer/gpu.js:538-556) of the context's Gaussians: an ArrayBuffer. */
  const saveSplat = () => serial(() => addon.saveSplat(ctx));

  const destroy = () => serial(() => addon.destroy(ctx));

  return { device: `cuda:${device}`, render, gradients, train, trainScene, lossGradientOf, forward, backward, loss, setTarget,
    getGaussians, loadPly, savePly, saveSplat, destroy };
}
