// antsApplyTransforms-compatible command line for displacement-field transforms, on the synx C ABI.
//
// The step right after the SyN stage: resample an image into the reference space through the
// fields antsRegistration wrote (prefix0Warp.nii.gz / prefix0InverseWarp.nii.gz).  Options follow
// Examples/antsApplyTransforms.cxx:1063-1240:
//   -d/--dimensionality 2|3      -i/--input image     -r/--reference-image image
//   -t/--transform file  (repeatable).  As in the reference's transform stack (:1183-1196), a
//       reference point is moved first by the LAST transform given, then by the one before it.
//       A displacement field image: [field,0] is accepted; [field,1] is rejected (a displacement
//       field has no closed-form inverse: pass the InverseWarp field instead).
//       A linear transform file (.mat / .txt, e.g. prefix0GenericAffine.mat; the types
//       synx_read_linear_transform reads): [file,1] applies its inverse.  A file holding several
//       transforms enters the stack in file order (reversed and each inverted for [file,1]).
//       HDF5 composite files (.h5) are not supported.
//   -n/--interpolation Linear (the default; other interpolators are rejected)
//   -f/--default-value v (0): value where the point maps outside the input image
//   -o/--output warped | [collapsed,1] | DisplacementField[collapsed]  (the collapsed form writes
//       the single displacement field equivalent to the stack, on the reference grid, :1115-1131)
//   --float 0|1 (computation is float32 either way)   -v/--verbose 0|1   --gpu N (not a reference option)
//
// GPU path: every field is brought onto the reference grid (synx_resample_field when its grid
// differs; a linear transform is written there as its displacement T(p) - p by
// synx_linear_field), the stack is composed in place, w <- w + u_i(x + w) from the last transform
// to the first (synx_compose), and the input is sampled once at x + w (synx_warp_image).  A
// displacement on the reference grid is zero outside it, so a transform that is not applied first
// acts as the identity where the transforms before it move a point off the reference grid (a
// linear transform applied first, the usual `-t warp -t affine` order, is exact everywhere).
#include "ants_apply_transforms.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "cli_common.h"
#include "nifti_io.h"
#include "synx.h"

namespace ants_b200 {
namespace {

using namespace cli;

bool same_grid(const synx_geom& a, const synx_geom& b) {
  for (int k = 0; k < 3; ++k)
    if (a.size[k] != b.size[k] || a.spacing[k] != b.spacing[k] || a.origin[k] != b.origin[k]) return false;
  for (int k = 0; k < 9; ++k)
    if (a.direction[k] != b.direction[k]) return false;
  return true;
}

struct DeviceBuffer {
  float* p = nullptr;
  explicit DeviceBuffer(size_t floats) { CLI_CK(cudaMalloc(&p, 4 * floats)); }
  ~DeviceBuffer() {
    if (p) cudaFree(p);
  }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
};

void step_ok(int rc, const char* what) {
  if (rc != 0) throw std::runtime_error(std::string(what) + ": " + synx_last_error(nullptr));
}

bool ends_with(const std::string& s, const std::string& suffix) {
  return s.size() >= suffix.size() && s.compare(s.size() - suffix.size(), suffix.size(), suffix) == 0;
}

// One transform of the stack: a displacement field image, or a linear transform of a .mat/.txt file.
struct StackEntry {
  std::string file;
  bool is_linear = false;
  bool invert = false;
  synx_linear linear{};
};

int run(const std::vector<std::string>& args, std::ostream& out) {
  std::map<std::string, std::vector<std::string>> opt;
  const std::map<std::string, std::string> alias = {
      {"-d", "dimensionality"}, {"-i", "input"},         {"-r", "reference-image"}, {"-t", "transform"},
      {"-n", "interpolation"},  {"-f", "default-value"}, {"-o", "output"},          {"-v", "verbose"},
      {"-e", "input-image-type"}, {"-u", "output-data-type"}, {"-h", "help"}};
  for (size_t i = 0; i < args.size(); ++i) {
    const std::string& k = args[i];
    std::string name;
    if (k.rfind("--", 0) == 0) name = k.substr(2);
    else if (alias.count(k)) name = alias.at(k);
    else throw std::runtime_error("unexpected argument '" + k + "'");
    if (name == "help") {
      out << "antsApplyTransforms_b200: antsApplyTransforms for displacement-field and linear transform stacks on a B200\n";
      return EXIT_SUCCESS;
    }
    if (i + 1 >= args.size()) throw std::runtime_error("option --" + name + " needs a value");
    opt[name].push_back(args[++i]);
  }
  auto one = [&](const std::string& n, const std::string& def) -> std::string {
    auto it = opt.find(n);
    return it == opt.end() ? def : it->second.back();
  };
  const int dim = std::atoi(one("dimensionality", "3").c_str());
  if (dim != 2 && dim != 3) throw std::runtime_error("--dimensionality must be 2 or 3");
  if (opt.count("input-image-type") && one("input-image-type", "0") != "0" &&
      lower(one("input-image-type", "scalar")) != "scalar")
    throw std::runtime_error("only scalar input images are supported");
  if (opt.count("interpolation") && lower(parse_call(one("interpolation", "Linear")).name) != "linear")
    throw std::runtime_error("only Linear interpolation is supported");
  if (!opt.count("reference-image")) throw std::runtime_error("a reference image (-r) is required");
  if (!opt.count("output")) throw std::runtime_error("an output (-o) is required");
  const bool verbose = one("verbose", "0") == "1" || lower(one("verbose", "0")) == "true";
  const int gpu = std::atoi(one("gpu", "0").c_str());
  const float defval = (float)std::atof(one("default-value", "0").c_str());

  // output form
  OptionCall o = parse_call(one("output", ""));
  bool collapse = false;
  std::string out_path;
  if (lower(o.name) == "displacementfield") {
    if (o.params.size() != 1) throw std::runtime_error("DisplacementField[file] needs one file name");
    collapse = true;
    out_path = o.params[0];
  } else if (o.name.empty() && !o.params.empty()) {
    out_path = o.params[0];
    collapse = o.params.size() > 1 && (o.params[1] == "1" || lower(o.params[1]) == "true");
    if (!collapse) throw std::runtime_error("-o [file,0] is not a supported output form");
  } else if (lower(o.name) == "linear" || lower(o.name) == "compositetransform") {
    throw std::runtime_error("-o " + o.name + "[...] is not supported (displacement fields only)");
  } else {
    out_path = o.name;
  }
  if (!collapse && !opt.count("input")) throw std::runtime_error("an input image (-i) is required");

  // transforms in command-line order
  std::vector<StackEntry> stack;
  for (const std::string& v : opt["transform"]) {
    OptionCall t = parse_call(v);
    std::string file = t.name;
    bool invert = false;
    if (file.empty()) {
      if (t.params.empty()) throw std::runtime_error("empty transform '" + v + "'");
      file = t.params[0];
      invert = t.params.size() > 1 && (t.params[1] == "1" || lower(t.params[1]) == "true");
    }
    if (lower(file) == "identity") continue;
    const std::string lf = lower(file);
    if (ends_with(lf, ".h5") || ends_with(lf, ".hdf5") || ends_with(lf, ".xfm"))
      throw std::runtime_error("transform '" + file + "': HDF5/composite transform files are not supported");
    if (ends_with(lf, ".mat") || ends_with(lf, ".txt")) {
      const int n = synx_read_linear_transform(file.c_str(), dim, 0, nullptr);
      if (n < 0) throw std::runtime_error(synx_last_error(nullptr));
      std::vector<StackEntry> part;
      for (int i = 0; i < n; ++i) {
        StackEntry e;
        e.file = file;
        e.is_linear = true;
        e.invert = invert;
        step_ok(synx_read_linear_transform(file.c_str(), dim, i, &e.linear) < 0 ? -1 : 0,
                "synx_read_linear_transform");
        part.push_back(e);
      }
      if (invert) std::reverse(part.begin(), part.end());
      stack.insert(stack.end(), part.begin(), part.end());
      continue;
    }
    if (invert)
      throw std::runtime_error("the inverse of displacement field '" + file +
                               "' is not available: use the inverse warp file antsRegistration wrote");
    StackEntry e;
    e.file = file;
    stack.push_back(e);
  }

  const nifti::Image ref = nifti::read(one("reference-image", ""));
  const synx_geom gr = to_geom(ref, dim);
  const long long N = gr.size[0] * gr.size[1] * gr.size[2];
  if (cudaSetDevice(gpu) != cudaSuccess) throw std::runtime_error("cannot use GPU " + std::to_string(gpu));

  // compose the stack on the reference grid: w = u_n, then w <- w + u_i(x + w), i = n-1 .. 1
  DeviceBuffer w((size_t)N * dim), tmp((size_t)N * dim);
  CLI_CK(cudaMemset(w.p, 0, 4 * (size_t)N * dim));
  for (int k = (int)stack.size() - 1; k >= 0; --k) {
    const StackEntry& e = stack[k];
    std::string note;
    // this transform's displacement on the reference grid, in tmp
    if (e.is_linear) {
      std::vector<float> u((size_t)N * dim);
      step_ok(synx_linear_field(&e.linear, e.invert ? 1 : 0, &gr, u.data()), "synx_linear_field");
      CLI_CK(cudaMemcpy(tmp.p, u.data(), 4 * (size_t)N * dim, cudaMemcpyHostToDevice));
      note = e.invert ? " (linear, inverse)" : " (linear)";
    } else {
      const nifti::Image f = nifti::read(e.file);
      if (f.components != dim || f.dim != dim)
        throw std::runtime_error("'" + e.file + "' is not a " + std::to_string(dim) + "-D displacement field");
      const synx_geom gf = to_geom(f, dim);
      const long long Nf = f.voxels();
      if (same_grid(gf, gr)) {
        CLI_CK(cudaMemcpy(tmp.p, f.data.data(), 4 * (size_t)N * dim, cudaMemcpyHostToDevice));
      } else {
        DeviceBuffer src((size_t)Nf * dim);
        CLI_CK(cudaMemcpy(src.p, f.data.data(), 4 * (size_t)Nf * dim, cudaMemcpyHostToDevice));
        step_ok(synx_resample_field(src.p, &gf, tmp.p, &gr, nullptr), "synx_resample_field");
        note = " (resampled)";
      }
    }
    if (k == (int)stack.size() - 1) {
      std::swap(w.p, tmp.p);
    } else {
      step_ok(synx_compose(tmp.p, w.p, &gr, 1.0f, w.p, nullptr), "synx_compose");
    }
    if (verbose) out << "  transform " << k << ": " << e.file << note << "\n";
  }

  if (collapse) {
    nifti::Image fo;
    fo.dim = dim;
    fo.components = dim;
    for (int k = 0; k < 3; ++k) {
      fo.size[k] = gr.size[k];
      fo.spacing[k] = gr.spacing[k];
      fo.origin[k] = gr.origin[k];
    }
    for (int k = 0; k < 9; ++k) fo.direction[k] = gr.direction[k];
    fo.data.resize((size_t)N * dim);
    CLI_CK(cudaMemcpy(fo.data.data(), w.p, 4 * (size_t)N * dim, cudaMemcpyDeviceToHost));
    nifti::write(out_path, fo);
    if (verbose) out << "wrote the collapsed displacement field " << out_path << "\n";
    return EXIT_SUCCESS;
  }

  nifti::Image in = nifti::read(one("input", ""));
  if (in.components != 1) throw std::runtime_error("the input must be a scalar image");
  const synx_geom gi = to_geom(in, dim);
  // a default value v outside the input: sample (I - v) with 0 outside and add v back (inside the
  // buffer the linear weights sum to one, so the result there is the sample of I)
  if (defval != 0.0f)
    for (float& x : in.data) x -= defval;
  const long long Ni = in.voxels();
  DeviceBuffer di((size_t)Ni), dout((size_t)N);
  CLI_CK(cudaMemcpy(di.p, in.data.data(), 4 * (size_t)Ni, cudaMemcpyHostToDevice));
  step_ok(synx_warp_image(di.p, &gi, w.p, &gr, dout.p, nullptr), "synx_warp_image");
  nifti::Image res = ref;
  res.components = 1;
  res.data.resize((size_t)N);
  CLI_CK(cudaMemcpy(res.data.data(), dout.p, 4 * (size_t)N, cudaMemcpyDeviceToHost));
  if (defval != 0.0f)
    for (float& x : res.data) x += defval;
  nifti::write(out_path, res);
  if (verbose) out << "wrote " << out_path << " (" << stack.size() << " transforms)\n";
  return EXIT_SUCCESS;
}

}  // namespace

int antsApplyTransforms(std::vector<std::string> args, std::ostream* out) {
  std::ostream& os = out ? *out : std::cout;
  try {
    return run(args, os);
  } catch (const std::exception& e) {
    std::cerr << "antsApplyTransforms_b200: " << e.what() << std::endl;
    return EXIT_FAILURE;
  }
}

}  // namespace ants_b200

int main(int argc, char** argv) {
  std::vector<std::string> args(argv + 1, argv + argc);
  return ants_b200::antsApplyTransforms(args, &std::cout);
}
