// antsApplyTransforms-compatible command line for displacement-field and linear transforms, on the
// synx C ABI.
//
// The step right after the SyN stage: resample an image into the reference space through the
// fields antsRegistration wrote (prefix0Warp.nii.gz / prefix0InverseWarp.nii.gz) and the linear
// transforms before them (prefix0GenericAffine.mat).  Options follow
// Examples/antsApplyTransforms.cxx:1063-1240:
//   -d/--dimensionality 2|3      -i/--input image     -r/--reference-image image
//   --time-index t (with -e 3: volume t alone, into a 3-D image)   -z/--static-cast-for-R (accepted)
//   Unknown options are accepted with a warning, as the reference's parser keeps and ignores them.
//   -e/--input-image-type 0|scalar (default) | 3|time-series | 4|multichannel (each volume or channel
//       resampled in turn)
//   -t/--transform file  (repeatable).  Order: a reference point is moved by the FIRST transform
//       given, then by the second, and so on; the input is sampled where the last one puts it.
//       This is the reference's order: its parser stores repeated options newest first
//       (Utilities/antsCommandLineOption.cxx:42,64 push_front), the transform loop adds them to
//       an ITK composite in that stored order (Examples/itkantsRegistrationHelper.h:1284-1459),
//       and a composite applies the transform added last first.  So `-t 1Warp -t 0GenericAffine.mat`
//       maps p to A(p + u(p)), as the registration's own composite does.
//       A displacement field image: [field,0] is accepted; [field,1] is rejected (a displacement
//       field has no closed-form inverse: pass the InverseWarp field instead).
//       A linear transform file (.mat / .txt / .tfm; the types synx_read_linear_transform reads): [file,1]
//       applies its inverse.  The transforms of one file act as the composite the file holds: the
//       last one first, or for [file,1] the inverse of the first one first (:1440-1451).
//       A composite transform in ITK's text form (.txt holding displacement fields, as
//       antsRegistration_b200 -a 1 writes prefixComposite.txt) acts as its entries, the last one
//       first; [composite,1] is rejected when it holds fields.  HDF5 composite files (.h5) are not
//       supported.
//   -n/--interpolation Linear (the default) | NearestNeighbor | GenericLabel[Linear] (label images;
//       others are rejected)
//   -f/--default-value v (0): value where the point maps outside the input image
//   -o/--output warped | [warped,0] | [collapsed,1] | DisplacementField[collapsed]  (the collapsed
//       form writes the single displacement field equivalent to the stack, on the reference grid,
//       :1115-1131) | CompositeTransform[file.txt]  (the stack uncollapsed, in ITK's text form; no
//       reference image needed)
//       | Linear[collapsed.mat,invert]  (an all-linear stack as one affine transform file)
//   -u/--output-data-type char|uchar|short|int|float|double|default (a cast of the float result)
//   --float 0|1 (computation is float32 either way; output files, the collapsed field and the
//       default output type, are float64 unless --float 1, as the reference writes them)
//   -v/--verbose 0|1   --gpu N (not a reference option)
//
// GPU path.  The chain of transforms, in application order, is split into a leading run of
// linear transforms L_pre, a middle part from the first field to the last field, and a trailing
// run of linear transforms L_post (a chain without fields is all L_pre).  The linear ends are
// folded into grid geometry, which the device functions take as general index <-> physical maps:
//   * the evaluation grid G has the reference grid's voxels at L_pre(p) (direction M*D, origin
//     M*o + b for L_pre(p) = M p + b);
//   * the input image is given the geometry under which sampling at q reads it at L_post(q).
// The middle part is composed on G, each transform acting on the current point x_G + w:
//   * the first field: sampled on its own grid at G's points (a copy when its grid is G);
//   * a later field on G: w <- w + d(x + w) (synx_compose);
//   * a later field on another grid: d sampled on its own grid at x + w, one component at a time
//     (synx_warp_image), then w <- d(x + w) + w (synx_field_affine_update);
//   * a linear transform T(p) = A p + b: w <- (T(x) - x) + A w (synx_linear_field, then
//     synx_field_affine_update).
// The input is sampled once at L_post(x_G + w) (synx_warp_image).  Every transform is therefore
// applied at the point itself, with one interpolation per field and the interpolators' own rule
// outside a field's grid (no displacement), as ITK's composite applies them.  The collapsed field,
// L_post(x_G + w) - p, is assembled on the host while it is written.
#include "ants_apply_transforms.h"
#include "antsApplyTransforms.h"  // the exported ants::antsApplyTransforms

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "cli_common.h"
#include "composite_txt.h"
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

// One transform of the chain, in application order.
struct ChainItem {
  std::string file;
  bool is_linear = false;
  Map map;  // linear transforms
  synx_linear linear{};
  bool invert = false;
  // a displacement field read from a composite file: component planes on its own grid (a field
  // given as an image file is read when its turn comes)
  bool in_memory = false;
  std::vector<float> planes;
  synx_geom grid{};
};

// The entries of a text composite file in application order (the last entry first), or an empty
// list when the file holds no displacement field (a linear file, read by the linear reader) or is
// not a composite the text reader takes.
std::vector<ChainItem> composite_chain(const std::string& file, int dim, bool invert) {
  std::vector<composite::Item> items;
  try {
    items = composite::read(file);
  } catch (const std::exception&) {
    // not a composite the text reader takes: the linear reader reports on it, unless it names a
    // displacement field, whose own error is the one to report
    std::ifstream in(file, std::ios::binary);
    const std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    if (text.find("DisplacementFieldTransform_") != std::string::npos) throw;
    return {};
  }
  if (std::none_of(items.begin(), items.end(), [](const composite::Item& it) { return it.is_field(); })) return {};
  if (invert)
    throw std::runtime_error("the inverse of composite transform '" + file +
                             "' is not available: it holds displacement fields (use the inverse composite)");
  std::vector<ChainItem> chain;
  for (auto it = items.rbegin(); it != items.rend(); ++it) {
    ChainItem c;
    c.file = file;
    if (it->is_field()) {
      c.grid = composite::field_geom(*it, dim);
      const size_t n = it->field.size() / (size_t)dim;
      c.planes.resize(it->field.size());
      for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < dim; ++k) c.planes[(size_t)k * n + i] = it->field[i * (size_t)dim + (size_t)k];
      c.in_memory = true;
    } else {
      c.is_linear = true;
      c.linear = composite::to_linear(*it, dim);
      c.map = map_of(c.linear, false);
    }
    chain.push_back(std::move(c));
  }
  return chain;
}

int run(const std::vector<std::string>& args, std::ostream& out) {
  std::map<std::string, std::vector<std::string>> opt;
  const std::map<std::string, std::string> alias = {
      {"-d", "dimensionality"}, {"-i", "input"},         {"-r", "reference-image"}, {"-t", "transform"},
      {"-n", "interpolation"},  {"-f", "default-value"}, {"-o", "output"},          {"-v", "verbose"},
      {"-e", "input-image-type"}, {"-u", "output-data-type"}, {"-h", "help"}, {"-z", "static-cast-for-R"}};
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
  // input image type (:1053-1069): scalar, or multichannel / time series, whose channels or volumes
  // are resampled one by one (:516-535, :903-981); vector and tensor inputs are rejected
  const std::string itype = lower(one("input-image-type", "0"));
  const bool multichannel = itype == "4" || itype == "multichannel";
  bool series = itype == "3" || itype == "time-series";
  if (!(itype == "0" || itype == "scalar" || multichannel || series))
    throw std::runtime_error("only scalar (0), time-series (3) and multichannel (4) input images are supported");
  if (series && dim != 3) throw std::runtime_error("time-series input (-e 3) needs -d 3");
  // --time-index t with -e 3: only volume t is resampled, into a 3-D image (:242-249, :283-317); the
  // reference reads it for time series only
  long long time_index = -1;
  if (series && opt.count("time-index")) {
    const std::string v = one("time-index", "0");
    char* end = nullptr;
    time_index = std::strtoll(v.c_str(), &end, 10);
    if (end == v.c_str() || *end != '\0' || time_index < 0)
      throw std::runtime_error("--time-index must be a non-negative integer");
  }
  // options of the reference this front end keeps without using (-z only changes how R reads
  // transforms) or does not know: the reference's parser keeps unknown options and goes on
  // (Utilities/antsCommandLineParser.cxx:124-160); this one names them on stderr
  static const char* const known[] = {"dimensionality", "input-image-type", "time-index", "input", "reference-image",
                                      "output", "interpolation", "output-data-type", "transform", "default-value",
                                      "static-cast-for-R", "float", "verbose", "gpu"};
  for (const auto& kv : opt)
    if (std::find_if(std::begin(known), std::end(known), [&](const char* k) { return kv.first == k; }) ==
        std::end(known))
      std::cerr << "antsApplyTransforms_b200: WARNING: unknown option --" << kv.first << " ignored" << std::endl;
  const OptionCall icall = parse_call(one("interpolation", "Linear"));
  const std::string interp = lower(icall.name);
  if (interp != "linear" && interp != "nearestneighbor" && interp != "genericlabel")
    throw std::runtime_error("only Linear, NearestNeighbor and GenericLabel[Linear] interpolation are supported");
  if (interp == "genericlabel" && !icall.params.empty() && lower(icall.params[0]) != "linear")
    throw std::runtime_error("GenericLabel supports the Linear interpolator only");
  const bool nearest = interp == "nearestneighbor", label = interp == "genericlabel";
  if (!opt.count("output")) throw std::runtime_error("an output (-o) is required");
  const std::string out_form = lower(parse_call(one("output", "")).name);
  const bool linear_out = out_form == "linear";
  // Linear[...] and CompositeTransform[...] write transforms only (:436-460)
  if (!linear_out && out_form != "compositetransform" && !opt.count("reference-image"))
    throw std::runtime_error("a reference image (-r) is required");
  const bool verbose = one("verbose", "0") == "1" || lower(one("verbose", "0")) == "true";
  const int gpu = std::atoi(one("gpu", "0").c_str());
  const float defval = (float)std::atof(one("default-value", "0").c_str());
  // the reference computes in double unless --float 1 (:1237-1240, :1384-1405); its collapsed field and
  // the "default" output type are that type, so the files here are float64 unless --float 1 (the values
  // are computed in float either way)
  const std::string fl = lower(one("float", "0"));
  const int real_type = (fl == "1" || fl == "true") ? 16 : 64;
  // output pixel type of the warped image (:1168-1181, :1460-1520): a cast of the float result
  const std::map<std::string, int> out_types = {{"char", 256}, {"uchar", 2}, {"short", 4},     {"int", 8},
                                                {"float", 16}, {"double", 64}, {"default", real_type}};
  const std::string out_type = lower(one("output-data-type", "default"));
  if (!out_types.count(out_type))
    throw std::runtime_error("--output-data-type must be char, uchar, short, int, float, double or default");

  // output form
  OptionCall o = parse_call(one("output", ""));
  bool collapse = false, composite_out = false;
  std::string out_path;
  if (lower(o.name) == "displacementfield") {
    if (o.params.size() != 1) throw std::runtime_error("DisplacementField[file] needs one file name");
    collapse = true;
    out_path = o.params[0];
  } else if (o.name.empty() && !o.params.empty()) {
    out_path = o.params[0];
    // [file,1]: the collapsed field; [file,0]: the warped image, as a plain name (:404-421)
    collapse = o.params.size() > 1 && (o.params[1] == "1" || lower(o.params[1]) == "true");
  } else if (linear_out) {
    if (o.params.empty() || o.params.size() > 2) throw std::runtime_error("Linear[file.mat,invert] needs a file name");
    out_path = o.params[0];
  } else if (lower(o.name) == "compositetransform") {
    // the stack as one composite transform file, uncollapsed (:444-460, :690-701)
    if (o.params.size() != 1) throw std::runtime_error("CompositeTransform[file] needs one file name");
    composite_out = true;
    out_path = o.params[0];
  } else {
    out_path = o.name;
  }
  if (!collapse && !linear_out && !composite_out && !opt.count("input"))
    throw std::runtime_error("an input image (-i) is required");

  // the chain in application order: command-line order, each file's transforms as its composite
  std::vector<ChainItem> chain;
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
      throw std::runtime_error("transform '" + file +
                               "': HDF5 and MINC transform files are not supported (text composites .txt/.tfm are)");
    if (ends_with(lf, ".txt") || ends_with(lf, ".tfm")) {
      std::vector<ChainItem> cc = composite_chain(file, dim, invert);
      if (!cc.empty()) {
        for (ChainItem& c : cc) chain.push_back(std::move(c));
        continue;
      }
    }
    if (ends_with(lf, ".mat") || ends_with(lf, ".txt") || ends_with(lf, ".tfm")) {
      for (const LinearItem& li : read_linear_file(file, dim, invert)) {
        ChainItem c;
        c.file = file;
        c.is_linear = true;
        c.invert = invert;
        c.linear = li.linear;
        c.map = li.map;
        chain.push_back(c);
      }
      continue;
    }
    if (invert)
      throw std::runtime_error("the inverse of displacement field '" + file +
                               "' is not available: use the inverse warp file antsRegistration wrote");
    ChainItem c;
    c.file = file;
    chain.push_back(c);
  }

  if (linear_out) {
    // -o Linear[file.mat,invert] (:640-680): an all-linear stack collapsed into one affine, written as
    // an ITK transform file.  Like CollapseLinearTransforms (itkantsRegistrationHelper.hxx:3773-3825) the
    // center is that of the first transform that acts and has one; the inverse is written, as the
    // reference builds it, with the inverse matrix, offset -M^-1 b and center 0.  No device work.
    Map total;
    double center[3] = {0.0, 0.0, 0.0};
    bool have_center = false;
    for (const ChainItem& c : chain) {
      if (!c.is_linear)
        throw std::runtime_error("'" + c.file + "' is a displacement field: only linear stacks collapse to Linear[...]");
      total = mul(c.map, total);
      if (!have_center && c.linear.has_center) {
        for (int k = 0; k < 3; ++k) center[k] = c.linear.center[k];
        have_center = true;
      }
    }
    synx_linear t;
    if (o.params.size() > 1 && o.params[1] != "0" && lower(o.params[1]) != "false") {
      Map inv;
      if (!inverse(total, inv)) throw std::runtime_error("the collapsed linear transform is singular, no inverse");
      const double zero[3] = {0.0, 0.0, 0.0};
      t = linear_of(inv, dim, zero);
    } else {
      t = linear_of(total, dim, center);
    }
    step_ok(synx_write_linear_transform(out_path.c_str(), &t), "synx_write_linear_transform");
    if (verbose) out << "wrote the collapsed linear transform " << out_path << "\n";
    return EXIT_SUCCESS;
  }

  if (composite_out) {
    // ITK's queue order: the transform acting last first.  Linear entries in matrix-offset form
    // (AffineTransform: a rigid or similarity entry keeps its map, not its type); an inverted one as
    // its inverse map about the same center; fields with their own grids.  Text form only.
    std::vector<composite::Item> items;
    for (auto it = chain.rbegin(); it != chain.rend(); ++it) {
      const ChainItem& c = *it;
      if (c.is_linear) {
        items.push_back(composite::linear_item(c.invert ? linear_of(c.map, dim, c.linear.center) : c.linear, dim));
        continue;
      }
      synx_geom gf;
      std::vector<float> planes;
      if (c.in_memory) {
        gf = c.grid;
        planes = c.planes;
      } else {
        nifti::Image f = nifti::read(c.file);
        if (f.components != dim || f.dim != dim || f.time_series)
          throw std::runtime_error("'" + c.file + "' is not a " + std::to_string(dim) + "-D displacement field");
        gf = to_geom(f, dim);
        planes = std::move(f.data);
      }
      const size_t n = planes.size() / (size_t)dim;
      std::vector<float> v(planes.size());
      for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < dim; ++k) v[i * (size_t)dim + (size_t)k] = planes[(size_t)k * n + i];
      items.push_back(composite::field_item(gf, v, real_type == 64));
    }
    composite::write(out_path, dim, items);
    if (verbose) out << "wrote the composite transform " << out_path << "\n";
    return EXIT_SUCCESS;
  }

  // split: leading linear run, middle (first field .. last field), trailing linear run
  size_t first_field = chain.size(), last_field = chain.size();
  for (size_t k = 0; k < chain.size(); ++k)
    if (!chain[k].is_linear) {
      if (first_field == chain.size()) first_field = k;
      last_field = k;
    }
  Map pre, post;
  const size_t lead_end = first_field;  // [0, lead_end) folds into the evaluation grid
  const size_t tail_begin = first_field == chain.size() ? chain.size() : last_field + 1;
  for (size_t k = 0; k < lead_end; ++k) pre = mul(chain[k].map, pre);
  for (size_t k = tail_begin; k < chain.size(); ++k) post = mul(chain[k].map, post);

  const nifti::Image ref = nifti::read(one("reference-image", ""));
  const synx_geom gr = to_geom(ref, dim);
  const long long N = gr.size[0] * gr.size[1] * gr.size[2];
  const synx_geom ge = push_forward(gr, pre);  // the evaluation grid
  if (cudaSetDevice(gpu) != cudaSuccess) throw std::runtime_error("cannot use GPU " + std::to_string(gpu));

  // compose the middle part on the evaluation grid
  DeviceBuffer w((size_t)N * dim), tmp((size_t)N * dim);
  CLI_CK(cudaMemset(w.p, 0, 4 * (size_t)N * dim));
  for (size_t k = 0; k < chain.size(); ++k) {
    const ChainItem& c = chain[k];
    if (k < lead_end || k >= tail_begin) {
      if (verbose)
        out << "  transform " << k << ": " << c.file << (c.invert ? " (linear, inverse" : " (linear")
            << (k < lead_end ? ", folded into the evaluation grid)" : ", folded into the input geometry)") << "\n";
      continue;
    }
    std::string note;
    if (c.is_linear) {
      // after w: T(x + w) - x = (T(x) - x) + A w, exact wherever the point is
      std::vector<float> u((size_t)N * dim);
      step_ok(synx_linear_field(&c.linear, c.invert ? 1 : 0, &ge, u.data()), "synx_linear_field");
      CLI_CK(cudaMemcpy(tmp.p, u.data(), 4 * (size_t)N * dim, cudaMemcpyHostToDevice));
      step_ok(synx_field_affine_update(tmp.p, w.p, &ge, c.map.M, w.p, nullptr), "synx_field_affine_update");
      note = c.invert ? " (linear, inverse)" : " (linear)";
    } else {
      nifti::Image f;
      synx_geom gf;
      const float* fdata = nullptr;
      if (c.in_memory) {
        gf = c.grid;
        fdata = c.planes.data();
      } else {
        f = nifti::read(c.file);
        if (f.components != dim || f.dim != dim || f.time_series)
          throw std::runtime_error("'" + c.file + "' is not a " + std::to_string(dim) + "-D displacement field");
        gf = to_geom(f, dim);
        fdata = f.data.data();
      }
      const long long Nf = gf.size[0] * gf.size[1] * gf.size[2];
      if (same_grid(gf, ge)) {
        // on the evaluation grid: the first field is copied, a later one composed (w + d(x + w))
        CLI_CK(cudaMemcpy(k == first_field ? w.p : tmp.p, fdata, 4 * (size_t)N * dim, cudaMemcpyHostToDevice));
        if (k != first_field) step_ok(synx_compose(tmp.p, w.p, &ge, 1.0f, w.p, nullptr), "synx_compose");
      } else {
        DeviceBuffer src((size_t)Nf * dim);
        CLI_CK(cudaMemcpy(src.p, fdata, 4 * (size_t)Nf * dim, cudaMemcpyHostToDevice));
        if (k == first_field) {
          // sampled on its own grid at the evaluation grid's points
          step_ok(synx_resample_field(src.p, &gf, w.p, &ge, nullptr), "synx_resample_field");
        } else {
          // sampled on its own grid at x + w, one component at a time, then added: w + d(x + w)
          for (int cc = 0; cc < dim; ++cc)
            step_ok(synx_warp_image(src.p + (size_t)cc * Nf, &gf, w.p, &ge, tmp.p + (size_t)cc * N, nullptr),
                    "synx_warp_image");
          const double I3[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
          step_ok(synx_field_affine_update(tmp.p, w.p, &ge, I3, w.p, nullptr), "synx_field_affine_update");
        }
        note = " (own grid)";
      }
    }
    if (verbose) out << "  transform " << k << ": " << c.file << note << "\n";
  }

  if (collapse) {
    nifti::Image fo;
    fo.out_datatype = real_type;
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
    if (lead_end > 0 || tail_begin < chain.size()) {
      // displacement of reference voxel p: L_post(L_pre(p) + w) - p, component planes
      const long long nx = gr.size[0], ny = gr.size[1];
      for (long long i = 0; i < N; ++i) {
        const double idx[3] = {(double)(i % nx), (double)((i / nx) % ny), (double)(i / (nx * ny))};
        double p[3], q[3];
        for (int r = 0; r < 3; ++r) {
          p[r] = gr.origin[r];
          for (int c = 0; c < 3; ++c) p[r] += gr.direction[r * 3 + c] * gr.spacing[c] * idx[c];
        }
        for (int r = 0; r < 3; ++r) {
          q[r] = pre.b[r] + (r < dim ? fo.data[(size_t)r * N + i] : 0.0);
          for (int c = 0; c < 3; ++c) q[r] += pre.M[r * 3 + c] * p[c];
        }
        for (int r = 0; r < dim; ++r) {
          double s = post.b[r];
          for (int c = 0; c < 3; ++c) s += post.M[r * 3 + c] * q[c];
          fo.data[(size_t)r * N + i] = (float)(s - p[r]);
        }
      }
    }
    nifti::write(out_path, fo);
    if (verbose) out << "wrote the collapsed displacement field " << out_path << "\n";
    return EXIT_SUCCESS;
  }

  nifti::Image in = nifti::read(one("input", ""));
  if (series ? (in.components > 1 && !in.time_series) : multichannel ? in.time_series : in.components != 1)
    throw std::runtime_error(series ? "the input is not a time series (-e 3)"
                             : multichannel ? "the input is a time series (use -e 3)"
                             : "the input must be a scalar image (-e 3 resamples a time series, -e 4 a multichannel image)");
  if (time_index >= 0) {
    if (time_index >= in.components)
      throw std::runtime_error("time index to extract is out of range [0, " + std::to_string(in.components - 1) + "]");
    const long long nv = in.voxels();
    in.data.erase(in.data.begin() + (time_index + 1) * nv, in.data.end());
    in.data.erase(in.data.begin(), in.data.begin() + time_index * nv);
    in.components = 1;
    in.time_series = false;
    series = false;
  }
  const int channels = in.components;
  synx_geom gi = to_geom(in, dim);
  if (tail_begin < chain.size()) {
    // sampling at q reads the input at L_post(q): the input's grid pulled back by L_post
    Map back;
    if (!inverse(post, back)) throw std::runtime_error("the trailing linear transforms have a singular matrix");
    gi = push_forward(gi, back);
  }
  // a default value v outside the input: sample (I - v) with 0 outside and add v back (inside the
  // buffer the linear weights sum to one, so the result there is the sample of I)
  if (defval != 0.0f)
    for (float& x : in.data) x -= defval;
  const long long Ni = in.voxels();
  DeviceBuffer di((size_t)Ni), dout((size_t)N);
  nifti::Image res = ref;
  res.out_datatype = out_types.at(out_type);
  res.components = channels;
  res.time_series = series;
  res.time_step = in.time_step;
  res.data.resize((size_t)N * channels);
  for (int c = 0; c < channels; ++c) {  // one channel (component plane) at a time
    CLI_CK(cudaMemcpy(di.p, in.data.data() + (size_t)c * Ni, 4 * (size_t)Ni, cudaMemcpyHostToDevice));
    if (label) step_ok(synx_warp_image_label(di.p, &gi, w.p, &ge, dout.p, nullptr), "synx_warp_image_label");
    else if (nearest) step_ok(synx_warp_image_nearest(di.p, &gi, w.p, &ge, dout.p, nullptr), "synx_warp_image_nearest");
    else step_ok(synx_warp_image(di.p, &gi, w.p, &ge, dout.p, nullptr), "synx_warp_image");
    CLI_CK(cudaMemcpy(res.data.data() + (size_t)c * N, dout.p, 4 * (size_t)N, cudaMemcpyDeviceToHost));
  }
  if (defval != 0.0f)
    for (float& x : res.data) x += defval;
  nifti::write(out_path, res);
  if (verbose) out << "wrote " << out_path << " (" << chain.size() << " transforms)\n";
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

namespace ants {

int antsApplyTransforms(std::vector<std::string> args, std::ostream* out_stream) {
  return ants_b200::antsApplyTransforms(std::move(args), out_stream);
}

}  // namespace ants

#ifndef SYNX_CLI_NO_MAIN
int main(int argc, char** argv) {
  std::vector<std::string> args(argv + 1, argv + argc);
  return ants::antsApplyTransforms(args, &std::cout);
}
#endif
