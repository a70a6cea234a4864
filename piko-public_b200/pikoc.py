"""pikoc for B200: compiles a pipeline written against the reference's stage
interface -- a PikoPipe class header and its .pikostage files, unchanged --
into a shared library that runs it on the GPU.

    python piko-public_b200/pikoc.py PIPE_HEADER OUT_DIR [-D NAME[=VALUE] ...]

The reference's compiler (pikoc, clang/LLVM 3.2 based) analyses the pipe and
generates the pipe class's host methods and per-stage kernels
(pikoc/src/pikoc.cpp:69-318, pikoc/src/Backend/PTXBackend.cpp:741-1026).
Here:

* device code: the pipe header is compiled with NVRTC for sm_100a with
  `-default-device` (stage functions carry no __device__ annotation in the
  reference's files), `--fmad=false` (the reference's CPU backend does not
  contract), `__PIKOC_DEVICE__` defined and include/piko/ on the include path.
  A generated glue defines each stage's declared emit() (routing through
  piko::Stage::emit_impl) and two kernels per stage, piko_assign_<i> and
  piko_process_<i>, around the bodies of include/piko_stage_device.cuh.
* host code: a generated .cu defines the pipe class's allocate / prepare /
  run_single / run / destroy (declared by the reference's pipe header,
  rasterPipe.h:40-44) on piko::PipeCore (include/piko_stage.cuh), with
  `__PIKOC_HOST__` defined; the pipe's stage objects, linked by its own
  pikoConnect calls, are the stages the runtime launches.  The cubin is
  embedded.  The library also exports a small C ABI (pikoc_*) for tests and
  foreign callers.

Work is ordered and the screen resolved as the reference's one-thread CPU run
does (piko_stage.cuh), so the image equals the reference's.
"""
import ctypes
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.environ.get("NVCC", os.path.join(CUDA, "bin", "nvcc"))


class PikocError(RuntimeError):
    pass


# ------------------------------------------------------------------ parsing
def _strip_comments(text):
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def _block(text, start):
    """The text between the brace at or after `start` and its match."""
    i = text.index("{", start)
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[i + 1:j]
    raise PikocError("unbalanced braces")


def _sources(pipe_header):
    """Every header and stage file of the pipeline directory tree."""
    base = os.path.dirname(os.path.abspath(pipe_header))
    out = []
    for dirpath, _, files in os.walk(base):
        for f in files:
            if f.endswith((".h", ".hpp", ".pikostage")):
                out.append(os.path.join(dirpath, f))
    return out


def parse(pipe_header):
    """The pipe class, its stage members in declaration order, which stage
    classes declare their own emit(), and the parameter lists of the pipe's
    allocate and run declarations."""
    text = _strip_comments(open(pipe_header).read())
    m = re.search(r"class\s+(\w+)\s*:\s*public\s+PikoPipe", text)
    if not m:
        raise PikocError(f"{pipe_header}: no class derived from PikoPipe")
    pipe = m.group(1)
    body = _block(text, m.end())
    stages = {}
    for path in _sources(pipe_header):
        src = _strip_comments(open(path, errors="replace").read())
        for sm in re.finditer(r"class\s+(\w+)\s*:\s*public\s+Stage\s*<", src):
            cls = _block(src, sm.end())
            stages[sm.group(1)] = bool(re.search(r"\bvoid\s+emit\s*\(", cls))
    members = [(t, n) for t, n in re.findall(r"^\s*(\w+)\s+(\w+)\s*;", body, flags=re.M) if t in stages]
    if not members:
        raise PikocError(f"{pipe}: no stage members")
    params = {}
    for name in ("allocate", "run"):
        pm = re.search(r"\bvoid\s+" + name + r"\s*\(([^)]*)\)", body)
        if not pm:
            raise PikocError(f"{pipe}: no {name}() declaration")
        params[name] = " ".join(pm.group(1).split())
    im = re.match(r"ConstantState\s*&\s*(\w+)\s*,\s*MutableState\s*&\s*(\w+)\s*,\s*(\w+)\s*\*\s*(\w+)\s*,\s*int\s+(\w+)",
                  params["allocate"])
    if not im:
        raise PikocError(f"{pipe}: allocate() is not (ConstantState&, MutableState&, In*, int)")
    return {"pipe": pipe, "members": members, "own_emit": {t: stages[t] for t, _ in members},
            "params": params, "arg_names": im.groups()[:2] + im.groups()[3:], "input_type": im.group(3)}


# ------------------------------------------------------------------ generation
def device_source(info, header_name):
    lines = ["// generated by pikoc.py: device glue of " + info["pipe"],
             "#define __PIKOC_DEVICE__", "#define PIKO_COMPAT_API",
             f'#include "{header_name}"', ""]
    for i, (t, _) in enumerate(info["members"]):
        if info["own_emit"][t]:
            lines.append(f"void {t}::emit({t}::Out p, int port) {{ emit_impl(p, port); }}")
        lines += [
            f'extern "C" __global__ void piko_assign_{i}({t} stage, piko::detail::StageRun* run, const {t}::In* in, '
            f"unsigned n, int pass)",
            "{ piko::detail::assign_body(stage, run, in, n, pass); }",
            f'extern "C" __global__ void piko_process_{i}({t} stage, piko::detail::StageRun* run, const {t}::In* in, '
            "unsigned* work, piko::MutableState* ms, int pass, int mode)",
            "{ piko::detail::process_body(stage, run, in, work, ms, pass, mode); }", ""]
    return "\n".join(lines)


def host_source(info, header_path, cubin):
    p = info["pipe"]
    cs, ms, inp, cnt = info["arg_names"]
    n = len(info["members"])
    arr = ",".join(str(b) for b in cubin)
    out = [f"// generated by pikoc.py: host methods of {p} on piko::PipeCore",
           "#define __PIKOC_HOST__", "#define PIKO_COMPAT_API",
           "#define __PIKO_DEVICE_MEMBERS__ void* pikoc_rt_ = nullptr;",
           "#include <cstdio>", "#include <string>", "#include <vector>",
           f'#include "{header_path}"', '#include "piko_stage.cuh"', "",
           f"static const unsigned char kCubin[] = {{{arr}}};", "",
           "namespace {",
           "struct PikocRt {", "  piko::PipeCore core;", "  cudaLibrary_t lib = nullptr;",
           "  ~PikocRt() { core.destroy(); if (lib) cudaLibraryUnload(lib); }", "};",
           "void pikoc_check(cudaError_t e, const char* what)", "{",
           "  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + \": \" + cudaGetErrorString(e));",
           "}", "}  // namespace", "",
           "unsigned* PikoScreen::getData()", "{",
           "  if (!core_) return nullptr;",
           "  h_data_.resize((size_t)core_->width() * core_->height());",
           "  core_->getData(h_data_.data());", "  return h_data_.data();", "}", "",
           f"void {p}::allocate({info['params']['allocate']})", "{",
           f"  constState_ = &{cs};", f"  mutableState_ = &{ms};", f"  count_ = {cnt};",
           f"  h_input.copyFrom({inp}, {cnt});",
           "  destroy();",
           "  PikocRt* rt = new PikocRt();", "  pikoc_rt_ = rt;",
           "  pikoc_check(cudaLibraryLoadData(&rt->lib, kCubin, nullptr, nullptr, 0, nullptr, nullptr, 0), "
           "\"loading the stage kernels\");",
           f"  piko::StageCommon* objs[{n}] = {{{', '.join('&' + m for _, m in info['members'])}}};",
           f"  rt->core.specs.resize({n});"]
    for i, (t, m) in enumerate(info["members"]):
        out += ["  {", f"    piko::StageSpec& sp = rt->core.specs[{i}];",
                f"    sp.binX = {t}::kBinSizeX; sp.binY = {t}::kBinSizeY; sp.threads = {t}::kThreadsPerTile;",
                f"    sp.inSize = sizeof({t}::In); sp.outSize = sizeof({t}::Out); sp.objSize = sizeof({t});",
                f"    sp.obj = &{m};", "    cudaKernel_t k = nullptr;",
                f'    pikoc_check(cudaLibraryGetKernel(&k, rt->lib, "piko_assign_{i}"), "piko_assign_{i}");',
                "    sp.assignKernel = (const void*)k;",
                f'    pikoc_check(cudaLibraryGetKernel(&k, rt->lib, "piko_process_{i}"), "piko_process_{i}");',
                "    sp.processKernel = (const void*)k;",
                f"    const bool pixels = piko::detail::same_type<{t}::Out, Pixel>::value;",
                "    for (int port = 0; port < piko::kNumPorts; ++port) {",
                f"      void* to = objs[{i}]->outPort[port];",
                "      sp.links[port] = -2;",
                f"      for (int j = 0; j < {n}; ++j) if (to == (void*)objs[j]) sp.links[port] = j;",
                "      if (!to && pixels) sp.links[port] = piko::kScreen;   // Pixels go to PikoScreen",
                "    }", "  }"]
    out += [f"  rt->core.allocate({cs}, {ms}, h_input.getData(), {cnt});",
            "  pikoScreen.core_ = &rt->core;", "}", "",
            f"void {p}::prepare() {{ if (pikoc_rt_) static_cast<PikocRt*>(pikoc_rt_)->core.prepare(true); }}",
            f"void {p}::run_single() {{ if (pikoc_rt_) static_cast<PikocRt*>(pikoc_rt_)->core.run_single(); }}",
            f"void {p}::destroy()", "{", "  delete static_cast<PikocRt*>(pikoc_rt_);", "  pikoc_rt_ = nullptr;",
            "  pikoScreen.core_ = nullptr;", "}",
            # the reference's run() loops under GLUT; here it draws one frame
            f"void {p}::run({info['params']['run']})",
            "{", f"  allocate({cs}, {ms}, {inp}, {cnt});", "  prepare();", "  run_single();", "}", "",
            "// C ABI for tests and foreign callers: one pipe with its states",
            "namespace {",
            "struct PikocHandle {", f"  {p} pipe;", "  ConstantState cs{};", "  MutableState ms{};",
            "  std::vector<float> z;", "  std::string err;", "};", "}  // namespace", "",
            'extern "C" void* pikoc_new() { return new PikocHandle(); }',
            'extern "C" void pikoc_delete(void* h) { if (h) { static_cast<PikocHandle*>(h)->pipe.destroy(); '
            "delete static_cast<PikocHandle*>(h); } }",
            'extern "C" const char* pikoc_error(void* h) { return h ? static_cast<PikocHandle*>(h)->err.c_str() : ""; }',
            'extern "C" int pikoc_input_size() { return (int)sizeof(' + info["input_type"] + "); }",
            f'extern "C" int pikoc_stages() {{ return {n}; }}',
            "// W x H screen, column-major view-projection matrix, count input primitives",
            'extern "C" int pikoc_allocate(void* hv, int W, int H, const float* vp, const void* input, int count)', "{",
            "  PikocHandle* h = static_cast<PikocHandle*>(hv);",
            "  try {",
            "    h->cs = ConstantState{};", "    h->cs.screenSizeX = W; h->cs.screenSizeY = H;",
            "    h->cs.halfW = 0.5f * (float)W; h->cs.halfH = 0.5f * (float)H;",
            "    for (int i = 0; i < 16; ++i) h->cs.viewProjMatrix[i] = vp ? vp[i] : (i % 5 == 0 ? 1.0f : 0.0f);",
            "    h->z.assign((size_t)W * H, 1.0f);", "    h->ms.zBuffer = h->z.data();",
            f"    h->pipe.allocate(h->cs, h->ms, ({info['input_type']}*)input, count);",
            "    return 0;",
            "  } catch (const std::exception& e) { h->err = e.what(); return -1; }", "}",
            "// one frame: depth reset to 1.0 (as the reference's apps do before each frame), prepare, run_single",
            'extern "C" int pikoc_frame(void* hv)', "{",
            "  PikocHandle* h = static_cast<PikocHandle*>(hv);",
            "  try {", "    std::fill(h->z.begin(), h->z.end(), 1.0f);",
            "    h->pipe.prepare();", "    h->pipe.run_single();", "    return 0;",
            "  } catch (const std::exception& e) { h->err = e.what(); return -1; }", "}",
            'extern "C" int pikoc_read(void* hv, unsigned* fb, float* depth)', "{",
            "  PikocHandle* h = static_cast<PikocHandle*>(hv);",
            "  try {", "    const size_t n = (size_t)h->cs.screenSizeX * h->cs.screenSizeY;",
            "    if (fb) std::memcpy(fb, h->pipe.pikoScreen.getData(), n * 4);",
            "    PikocRt* rt = static_cast<PikocRt*>(h->pipe.pikoc_rt_);",
            "    if (depth && rt) pikoc_check(cudaMemcpy(depth, rt->core.device_depth(), n * 4, cudaMemcpyDeviceToHost), "
            '"depth");',
            "    return 0;",
            "  } catch (const std::exception& e) { h->err = e.what(); return -1; }", "}",
            'extern "C" int pikoc_processed(void* hv, unsigned long long* out, int n)', "{",
            "  PikocRt* rt = static_cast<PikocRt*>(static_cast<PikocHandle*>(hv)->pipe.pikoc_rt_);",
            "  if (!rt) return -1;", "  const auto& p = rt->core.processed();",
            "  for (int i = 0; i < n && i < (int)p.size(); ++i) out[i] = p[i];", "  return 0;", "}", ""]
    return "\n".join(out)


# ------------------------------------------------------------------ compilation
def _nvrtc():
    for name in (os.path.join(CUDA, "lib64", "libnvrtc.so.12"), "libnvrtc.so.12", "libnvrtc.so"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    raise PikocError("libnvrtc not found")


def nvrtc_cubin(source, name, options):
    """Compiles `source` with NVRTC; returns the cubin bytes (raises with the log)."""
    lib = _nvrtc()
    prog = ctypes.c_void_p()
    r = lib.nvrtcCreateProgram(ctypes.byref(prog), source.encode(), name.encode(), 0, None, None)
    if r != 0:
        raise PikocError(f"nvrtcCreateProgram: {r}")
    try:
        opts = [o.encode() for o in options]
        arr = (ctypes.c_char_p * len(opts))(*opts)
        r = lib.nvrtcCompileProgram(prog, len(opts), arr)
        size = ctypes.c_size_t()
        lib.nvrtcGetProgramLogSize(prog, ctypes.byref(size))
        log = ctypes.create_string_buffer(size.value + 1)
        lib.nvrtcGetProgramLog(prog, log)
        if r != 0:
            raise PikocError("NVRTC failed:\n" + log.value.decode(errors="replace"))
        lib.nvrtcGetCUBINSize(prog, ctypes.byref(size))
        buf = ctypes.create_string_buffer(size.value)
        if lib.nvrtcGetCUBIN(prog, buf) != 0:
            raise PikocError("nvrtcGetCUBIN failed")
        return buf.raw
    finally:
        lib.nvrtcDestroyProgram(ctypes.byref(prog))


def compile_pipe(pipe_header, out_dir, defines=(), verbose=False):
    """Builds OUT_DIR/libpikoc_<pipe>.so from the pipe header; returns its path."""
    pipe_header = os.path.abspath(pipe_header)
    info = parse(pipe_header)
    os.makedirs(out_dir, exist_ok=True)
    base = os.path.dirname(pipe_header)
    dev = device_source(info, os.path.basename(pipe_header))
    with open(os.path.join(out_dir, "device_glue.cu"), "w") as f:
        f.write(dev)
    opts = ["--gpu-architecture=sm_100a", "-default-device", "--fmad=false", "-std=c++17",
            f"-I{INCLUDE}", f"-I{os.path.join(INCLUDE, 'piko_nvrtc')}", f"-I{base}",
            f"-I{os.path.join(CUDA, 'include')}"] + [f"-D{d}" for d in defines]
    cubin = nvrtc_cubin(dev, "device_glue.cu", opts)
    host = host_source(info, pipe_header, cubin)
    src = os.path.join(out_dir, "host_glue.cu")
    with open(src, "w") as f:
        f.write(host)
    lib = os.path.join(out_dir, f"libpikoc_{info['pipe']}.so")
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "--fmad=false", "-std=c++17",
           "-Xcompiler", "-fPIC", "-shared", "-w", "-I", INCLUDE, "-I", base, "-o", lib + ".tmp", src]
    cmd += [f"-D{d}" for d in defines]
    if verbose:
        print(" ".join(cmd[:12]), "...")
    subprocess.run(cmd, check=True)
    os.replace(lib + ".tmp", lib)
    return lib


def main(argv):
    if len(argv) < 3:
        print(__doc__)
        return 2
    defines = []
    args = list(argv[1:])
    while "-D" in args:
        i = args.index("-D")
        defines.append(args[i + 1])
        del args[i:i + 2]
    print(compile_pipe(args[0], args[1], defines, verbose=True))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
