"""Host-side mirror of the reference's pipeline interface.

A reference application drives a pipeline like this
(pikoc/samples/rasterPipelineFixPt/main.cpp:99-232):

    RasterPipe piko_pipe;
    piko_pipe.allocate(constState, mutableState, triangleBuffer, nTris);
    ... per frame: resetDepthBuffer(); piko_pipe.prepare(); piko_pipe.run_single();
    unsigned* data = piko_pipe.pikoScreen.getData();
    piko_pipe.destroy();

The classes here keep those names, argument meanings and call order, and run
every stage on the GPU through libpiko_b200.so.  Differences a caller can see:
errors raise PikoError instead of exiting the process; the depth buffer is
reset to 1.0f and the colour buffer to the clear colour at the start of every
frame (the reference leaves the colour buffer of earlier frames in place,
which only differs when the camera moves between frames); and there is no
fixed 1024x768 limit on the depth buffer.
"""
import numpy as np

from . import runtime as rt

# raster_wtri under VTX_PRETRANSFORM (basicTypes/rasterTypes.h:8-34): Primitive
# {binID, launchIdx}, id, worldPos0..2 (screen x, y and depth), icol0..2 (ABGR)
raster_wtri = np.dtype([("binID", "<u4"), ("launchIdx", "<u4"), ("id", "<i4"),
                        ("worldPos0", "<f4", 3), ("worldPos1", "<f4", 3), ("worldPos2", "<f4", 3),
                        ("icol0", "<u4"), ("icol1", "<u4"), ("icol2", "<u4")])
assert raster_wtri.itemsize == 60

# piko_patch (reyesPipe/pikoTypes.h:65-73)
piko_patch = np.dtype([("binID", "<u4"), ("launchIdx", "<u4"), ("CP", "<f4", (16, 4)),
                       ("numSplits", "<i4"), ("nu", "<i4"), ("nv", "<i4"), ("id", "<i4"),
                       ("bbmin", "<f4", 2), ("bbmax", "<f4", 2)])
assert piko_patch.itemsize == 296


class ConstantState:
    """ConstantState (piko/builtinTypes.h:20-33) plus the light inputs of the
    host pre-transform (main.cpp:358-392)."""

    def __init__(self, screenSizeX=1024, screenSizeY=768):
        self.screenSizeX = screenSizeX
        self.screenSizeY = screenSizeY
        self.halfW = 0.5 * screenSizeX
        self.halfH = 0.5 * screenSizeY
        self.projMatrix = np.eye(4, dtype=np.float32).reshape(16)
        self.viewMatrix = np.eye(4, dtype=np.float32).reshape(16)
        self.viewProjMatrix = np.eye(4, dtype=np.float32).reshape(16)
        self.debX = self.debY = 0
        self.light_mode = 0
        self.light = (0.5773, 0.5773, 0.5773)
        self.eye = (0.0, 0.0, 0.0)

    def to_c(self):
        return rt.const_state(view_proj=self.viewProjMatrix, light_mode=self.light_mode, light=self.light,
                              eye=self.eye)


class MutableState:
    """MutableState (piko/builtinTypes.h:35-40): the depth buffer, sized to the
    screen instead of the reference's fixed 1024*768 floats.  After a frame it
    holds the frame's depth buffer."""

    def __init__(self, screenSizeX=1024, screenSizeY=768):
        self.zBuffer = np.ones(screenSizeX * screenSizeY, np.float32)


class PikoScreen:
    """The built-in drain stage (piko/stage.h:53-136)."""

    def __init__(self, pipe):
        self._pipe = pipe

    def getNumPixels(self):
        return self._pipe._scene.W * self._pipe._scene.H

    def getData(self):
        """RGBA8 words, R in the low byte, row 0 = bottom (pixel (x, y) at y*W + x)."""
        fb, depth = self._pipe._scene.read()
        self._pipe._last_depth = depth
        if self._pipe.mutableState_ is not None:
            self._pipe.mutableState_.zBuffer[: depth.size] = depth.reshape(-1)
        return fb.reshape(-1)


class _PipeBase:
    KIND = "raster"

    def __init__(self, ctx=None, **tuning):
        self._ctx = ctx if ctx is not None else rt.Context()
        self._pipe = rt.Pipe(self._ctx, self.KIND, **tuning)
        self._scene = None
        self._last_depth = None
        self.constState_ = None
        self.mutableState_ = None
        self.count_ = 0
        self.pikoScreen = PikoScreen(self)

    def prepare(self):
        """Re-reads constState (camera, light) for the next frames."""
        self._scene.prepare(self.constState_.to_c())

    def run_single(self):
        """One frame, synchronous like the generated run_single."""
        self._scene.run()
        self._scene.finish()

    def run(self, constState, mutableState, input, count):
        self.allocate(constState, mutableState, input, count)
        self.prepare()
        self.run_single()

    def destroy(self):
        if self._scene is not None:
            self._scene.close()
            self._scene = None
        self._pipe.close()

    def stats(self):
        return self._scene.stats()


class RasterPipe(_PipeBase):
    """RasterPipe (rasterPipe.h:16-45): VertexShaderStage -> RasterStage."""
    KIND = "raster"

    def allocate(self, constState, mutableState, input, count=None):
        """input: a raster_wtri array (the reference's pre-transformed input) or a
        scenes.RasterScene (world-space attributes, transformed on the device)."""
        self.constState_ = constState
        self.mutableState_ = mutableState
        W, H = constState.screenSizeX, constState.screenSizeY
        if isinstance(input, np.ndarray) and input.dtype == raster_wtri:
            n = len(input) if count is None else int(count)
            t = input[:n]
            xyz = np.concatenate([t["worldPos0"], t["worldPos1"], t["worldPos2"]], axis=1)
            icol = np.stack([t["icol0"], t["icol1"], t["icol2"]], axis=1)
            if n and not np.array_equal(t["id"], np.arange(n)):
                raise rt.PikoError(rt.ERR_INVALID, "raster_wtri ids must be 0..count-1 (loadTriangleBuffer order)")
            self._scene = rt.Scene(self._pipe, {"W": W, "H": H, "xyz": xyz, "icol": icol})
        else:
            if (input.W, input.H) != (W, H):
                raise rt.PikoError(rt.ERR_INVALID, "scene size differs from constState screen size")
            self._scene = rt.Scene(self._pipe, input)
            constState.viewProjMatrix = np.asarray(input.view_proj, np.float32)
            constState.light_mode = input.light_mode
            constState.light = tuple(float(v) for v in input.light)
            constState.eye = tuple(float(v) for v in input.eye)
        self.count_ = self._scene.N


class ReyesPipe(_PipeBase):
    """ReyesPipe (reyesPipe.h:12-40): Split (self loop) -> Dice -> Shade."""
    KIND = "reyes"

    def allocate(self, constState, mutableState, input, count=None):
        """input: a piko_patch array or a scenes.PatchScene."""
        self.constState_ = constState
        self.mutableState_ = mutableState
        W, H = constState.screenSizeX, constState.screenSizeY
        from .scenes import PatchScene
        if isinstance(input, np.ndarray) and input.dtype == piko_patch:
            n = len(input) if count is None else int(count)
            sc = PatchScene(W=W, H=H, patches=np.ascontiguousarray(input["CP"][:n], np.float32),
                            view_proj=np.asarray(constState.viewProjMatrix, np.float32))
        else:
            sc = input
            constState.viewProjMatrix = np.asarray(sc.view_proj, np.float32)
        self._scene = rt.Scene(self._pipe, sc)
        self.count_ = self._scene.N
