// antsRegistration-compatible command line for a single SyN + CC stage, on the synx C ABI.
//
// Accepted options (the reference's syntax, Examples/antsRegistration.cxx:30-548, parsed as in
// Examples/antsRegistrationTemplateHeader.h:545-651, :801-815, :1081-1087):
//   -d/--dimensionality 2|3        --float 0|1 (computation is float32 either way; the output files
//       are float32 with --float 1 and float64 by default, as the reference writes them)
//   -m/--metric CC[fixed,moving,weight,radius]
//   -t/--transform SyN[gradientStep,updateFieldVariance,totalFieldVariance]
//   -c/--convergence [NxNx...,threshold,window] or NxNx...
//   -f/--shrink-factors NxNx...     -s/--smoothing-sigmas NxNx...[vox|mm]
//   -o/--output prefix | [prefix,warpedImage,inverseWarpedImage]
//   -w/--winsorize-image-intensities [lower,upper]   -u/--use-histogram-matching 0|1
//   -v/--verbose 0|1   --random-seed N (accepted, no effect: the stage is deterministic)
//   -p/--print-similarity-measure-interval N, --write-interval-volumes N, -l/--use-estimate-learning-
//       rate-once (accepted; non-zero intervals are not implemented and draw a warning)
//   --minc 0 (1 is refused: NIfTI output only)   --version
//   Unknown options are accepted with a warning, as the reference's parser keeps and ignores them.
//   --gpu N (device index; not a reference option)
//   -r/--initial-moving-transform file | [file,useInverse] | identity | [fixed,moving,feature]
//       (repeatable, the first given acting first; linear .mat/.txt/.tfm files, or the translation derived
//       from two images: feature 0 geometric centers, 1 centers of mass, 2 origins)
//   -z/--collapse-output-transforms 0|1 (default 1)
//   -a/--write-composite-transform 0|1: prefixComposite.txt and prefixInverseComposite.txt instead of
//       the separate files, in ITK's text transform form (the reference writes .h5; HDF5 is not
//       available here)
//   -i/--initialize-transforms-per-stage 0|1 (needs -a 1 and -z 0)
//   -j/--save-state file.txt: the registration state (initial transforms, then the SyN stage's
//       fixed-to-middle and moving-to-middle fields each followed by its inverse; needs -a 1)
//   -k/--restore-state file.txt: a saved state; its linear transforms act as the initial moving
//       transform and, with -i 1, its four fields start the SyN stage (without -i the reference
//       makes the composed fields an initial displacement-field transform, which this stage does
//       not take: refused)
//   -x/--masks [fixedMask,movingMask] | fixedMask (metric masks; a name that is not a file = no mask)
// Output: prefix0Warp.nii.gz and prefix0InverseWarp.nii.gz (antsRegistrationTemplateHeader.cxx:74-90
// names for SyN); with initial transforms, prefix0GenericAffine.mat (them, collapsed) and
// prefix1Warp / prefix1InverseWarp, or without collapsing prefix<n>Warp after the n initial
// transforms; plus the warped images when requested.  The initial transform is folded into the
// moving image's geometry (an index <-> physical map the device functions take in general form),
// which samples the moving image at Init(x + psi_M(x)) exactly.  With -z 0, derived translations are
// written as prefix<n>DerivedInitialMovingTranslation.mat.  Other stages, metrics, initial fixed
// transforms and HDF5 transform files are rejected with EXIT_FAILURE.
#include "ants_registration.h"
#include "antsRegistration.h"  // the exported ants::antsRegistration

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "cli_common.h"
#include "composite_txt.h"
#include "nifti_io.h"
#include "synx.h"

namespace ants_b200 {
namespace {

using namespace cli;

nifti::Image like(const nifti::Image& geom_src, std::vector<float> data) {
  nifti::Image im = geom_src;
  im.components = 1;
  im.data = std::move(data);
  return im;
}

int run(const std::vector<std::string>& args, std::ostream& out) {
  std::map<std::string, std::vector<std::string>> opt;  // long name -> values in order
  const std::map<std::string, std::string> alias = {
      {"-d", "dimensionality"}, {"-m", "metric"}, {"-t", "transform"}, {"-c", "convergence"},
      {"-f", "shrink-factors"}, {"-s", "smoothing-sigmas"}, {"-o", "output"}, {"-v", "verbose"},
      {"-w", "winsorize-image-intensities"}, {"-u", "use-histogram-matching"}, {"-x", "masks"},
      {"-r", "initial-moving-transform"}, {"-q", "initial-fixed-transform"}, {"-n", "interpolation"},
      {"-a", "write-composite-transform"}, {"-z", "collapse-output-transforms"}, {"-h", "help"},
      {"-i", "initialize-transforms-per-stage"}, {"-j", "save-state"}, {"-k", "restore-state"},
      {"-p", "print-similarity-measure-interval"}, {"-l", "use-estimate-learning-rate-once"}};
  for (size_t i = 0; i < args.size(); ++i) {
    std::string k = args[i];
    std::string name;
    if (k.rfind("--", 0) == 0) name = k.substr(2);
    else if (alias.count(k)) name = alias.at(k);
    else throw std::runtime_error("unexpected argument '" + k + "'");
    if (name == "help") {
      out << "antsRegistrationSyN_b200: antsRegistration options for one SyN + CC stage on a B200\n";
      return EXIT_SUCCESS;
    }
    if (name == "version") {
      out << "antsRegistrationSyN_b200: the antsRegistration SyN + CC stage on the synx C ABI (sm_100a)\n";
      return EXIT_SUCCESS;
    }
    if (i + 1 >= args.size()) throw std::runtime_error("option --" + name + " needs a value");
    opt[name].push_back(args[++i]);
  }
  auto one = [&](const std::string& n, const std::string& def) -> std::string {
    auto it = opt.find(n);
    return it == opt.end() ? def : it->second.back();
  };
  for (const char* bad : {"initial-fixed-transform", "restrict-deformation"})
    if (opt.count(bad)) throw std::runtime_error(std::string("option --") + bad + " is not supported by this SyN+CC stage");
  // The reference's parser keeps options it does not know and goes on (Utilities/antsCommandLineParser
  // .cxx:124-160); so does this one, with a warning, since a misspelt option would otherwise pass unseen.
  // Options of the reference this stage does not implement: MINC output is refused (only NIfTI is
  // written); the full-scale metric printout (-p) and the interval volumes are ignored with a warning.
  static const char* const known[] = {
      "dimensionality", "output", "save-state", "restore-state", "write-composite-transform",
      "print-similarity-measure-interval", "write-interval-volumes", "collapse-output-transforms",
      "initialize-transforms-per-stage", "interpolation", "initial-moving-transform", "metric", "transform",
      "convergence", "smoothing-sigmas", "shrink-factors", "use-histogram-matching", "use-estimate-learning-rate-once",
      "winsorize-image-intensities", "masks", "float", "minc", "random-seed", "verbose", "gpu"};
  for (const auto& kv : opt) {
    if (std::find_if(std::begin(known), std::end(known), [&](const char* k) { return kv.first == k; }) ==
        std::end(known))
      std::cerr << "antsRegistrationSyN_b200: WARNING: unknown option --" << kv.first << " ignored" << std::endl;
  }
  for (const char* ignored : {"print-similarity-measure-interval", "write-interval-volumes"}) {
    if (!opt.count(ignored)) continue;
    const std::string v = opt[ignored].back();
    if (!(v == "0" || v.empty()))
      std::cerr << "antsRegistrationSyN_b200: WARNING: --" << ignored << " " << v << " is not implemented; ignored"
                << std::endl;
  }
  if (opt.count("minc")) {
    const std::string v = lower(opt["minc"].back());
    if (!(v == "0" || v == "false")) throw std::runtime_error("MINC output (--minc 1) is not supported: NIfTI only");
  }
  auto flag = [&](const std::string& n, bool def) {
    if (!opt.count(n)) return def;
    const std::string v = lower(one(n, ""));
    return !(v == "0" || v == "false");
  };
  // the reference's option checks (Examples/antsRegistration.cxx:629-655,
  // Examples/antsRegistrationTemplateHeader.h:154-172, :293-305)
  const bool composite_out = flag("write-composite-transform", false);
  const bool collapse = flag("collapse-output-transforms", true);
  const bool init_per_stage = flag("initialize-transforms-per-stage", false);
  const std::string save_state = opt.count("save-state") ? one("save-state", "") : "";
  const std::string restore_state = opt.count("restore-state") ? one("restore-state", "") : "";
  if (init_per_stage && !composite_out)
    throw std::runtime_error("--initialize-transforms-per-stage requires --write-composite-transform");
  if (!save_state.empty() && !composite_out) throw std::runtime_error("--save-state requires --write-composite-transform");
  if (init_per_stage && collapse)
    throw std::runtime_error("initialize-transforms-per-stage & collapse-output-transforms options are mutually exclusive");
  if (!restore_state.empty() && opt.count("initial-moving-transform"))
    throw std::runtime_error("restore-state option is mutually exclusive with initial-moving-transform & "
                             "initial-fixed-transform options");
  const bool histogram_matching = flag("use-histogram-matching", false);
  if (opt.count("interpolation") && lower(one("interpolation", "Linear")) != "linear")
    throw std::runtime_error("only Linear interpolation is supported for the warped outputs");

  const int dim = std::atoi(one("dimensionality", "3").c_str());
  if (dim != 2 && dim != 3) throw std::runtime_error("--dimensionality must be 2 or 3");
  // The reference computes in double unless --float 1 (antsRegistration.cxx:488-491, :707-722).
  // This stage computes in float32 (FP64 only in the CC window sums and the global reductions),
  // so a double request is honoured for the written files only, and said so on stderr.
  const bool use_float = flag("float", false);
  if (!use_float)
    std::cerr << "antsRegistrationSyN_b200: WARNING: double precision requested (--float 0, the reference's "
                 "default); this stage computes in float32 and writes its results widened to float64. Pass "
                 "--float 1 to request float32 explicitly."
              << std::endl;
  const bool verbose = one("verbose", "0") == "1" || lower(one("verbose", "0")) == "true";

  // initial moving transforms: linear files (or identity), in the order they act on a point (the
  // first -r given first, as antsApplyTransforms orders -t); the moving image is sampled at
  // Init(x + psi_M(x)), the composite ITK's SyN builds from the stored initial transforms and the
  // moving half-field
  std::vector<LinearItem> init;
  std::vector<std::pair<int, synx_linear>> derived;  // (stored option index, transform) of [fixed,moving,feature]
  const int n_init = (int)opt["initial-moving-transform"].size();
  for (int j = 0; j < n_init; ++j) {
    const std::string& v = opt["initial-moving-transform"][j];
    OptionCall r = parse_call(v);
    if (r.params.size() > 2) {
      // [fixed,moving,feature]: a translation derived from the two images (host arithmetic)
      const int feature = std::atoi(r.params[2].c_str());
      const nifti::Image a = nifti::read(r.params[0]);
      const nifti::Image b = nifti::read(r.params[1]);
      if (a.components != 1 || b.components != 1) throw std::runtime_error("scalar images expected in " + v);
      const synx_geom ga = to_geom(a, dim), gb = to_geom(b, dim);
      LinearItem li;
      if (synx_initial_translation(a.data.data(), &ga, b.data.data(), &gb, feature, &li.linear) != 0)
        throw std::runtime_error(std::string("synx_initial_translation: ") + synx_last_error(nullptr));
      li.map = map_of(li.linear, false);
      init.push_back(li);
      // the reference stores repeated options newest first and names the file by that index
      derived.emplace_back(n_init - 1 - j, li.linear);
      continue;
    }
    std::string file = r.name.empty() ? (r.params.empty() ? "" : r.params[0]) : r.name;
    const bool invert = r.name.empty() && r.params.size() > 1 && (r.params[1] == "1" || lower(r.params[1]) == "true");
    if (lower(file) == "identity") {
      LinearItem li;
      std::memset(&li.linear, 0, sizeof(li.linear));
      li.linear.dim = dim;
      li.linear.has_center = 1;  // the reference's identity is a MatrixOffsetTransformBase
      li.linear.matrix[0] = li.linear.matrix[4] = li.linear.matrix[8] = 1.0;
      init.push_back(li);
      continue;
    }
    const std::string lf = lower(file);
    const bool is_linear_file = lf.size() > 4 && (lf.compare(lf.size() - 4, 4, ".mat") == 0 ||
                                                  lf.compare(lf.size() - 4, 4, ".txt") == 0 ||
                                                  lf.compare(lf.size() - 4, 4, ".tfm") == 0);
    if (!is_linear_file)
      throw std::runtime_error("initial moving transform '" + file +
                               "': only linear transform files (.mat/.txt/.tfm) are supported");
    if (lf.compare(lf.size() - 4, 4, ".mat") != 0) {
      // a text composite holding displacement fields (prefixComposite.txt): the stage samples the moving
      // image through linear initial transforms only
      bool has_field = false;
      try {
        for (const composite::Item& it : composite::read(file)) has_field = has_field || it.is_field();
      } catch (const std::exception&) {
        // not a composite the text reader takes: the linear reader reports on it
      }
      if (has_field)
        throw std::runtime_error("initial moving transform '" + file +
                                 "' holds a displacement field: only linear initial transforms are supported");
    }
    for (const LinearItem& li : read_linear_file(file, dim, invert)) init.push_back(li);
  }
  // --restore-state: [linear..., fixedToMiddle, its inverse, movingToMiddle, its inverse]
  // (itkantsRegistrationHelper.hxx:3637-3725); a composite lists first the transform that acts last
  std::vector<composite::Item> state_fields;
  if (!restore_state.empty()) {
    std::vector<composite::Item> items = composite::read(restore_state);
    const size_t n = items.size();
    if (n >= 4 && items[n - 1].is_field() && items[n - 2].is_field() && items[n - 3].is_field() &&
        items[n - 4].is_field()) {
      if (!init_per_stage)
        throw std::runtime_error("--restore-state with SyN fields needs --initialize-transforms-per-stage 1 here: "
                                 "without it the reference starts from the composed fields as an initial "
                                 "displacement-field transform, which this stage does not take");
      state_fields.assign(items.end() - 4, items.end());
      items.resize(n - 4);
    }
    for (auto it = items.rbegin(); it != items.rend(); ++it) {
      if (it->is_field())
        throw std::runtime_error("--restore-state: displacement fields other than a SyN state are not supported");
      LinearItem li;
      li.linear = composite::to_linear(*it, dim);
      li.map = map_of(li.linear, false);
      init.push_back(li);
    }
  }
  Map init_map;
  double init_center[3] = {0.0, 0.0, 0.0};
  bool have_center = false;
  for (const LinearItem& li : init) {
    init_map = mul(li.map, init_map);
    // collapsing keeps the center of the transform that acts first and has one
    // (itkantsRegistrationHelper.hxx:3787-3798 scans the composite queue from its end)
    if (!have_center && li.linear.has_center) {
      for (int k = 0; k < 3; ++k) init_center[k] = li.linear.center[k];
      have_center = true;
    }
  }
  Map init_inverse;
  if (!inverse(init_map, init_inverse)) throw std::runtime_error("the initial moving transform is singular");
  const int gpu = std::atoi(one("gpu", "0").c_str());
  if (opt["transform"].size() != 1 || opt["metric"].size() != 1)
    throw std::runtime_error("exactly one stage (one --transform and one --metric) is supported");
  OptionCall t = parse_call(opt["transform"][0]);
  if (lower(t.name) != "syn") throw std::runtime_error("only the SyN transform is supported, got '" + t.name + "'");
  OptionCall m = parse_call(opt["metric"][0]);
  if (lower(m.name) != "cc") throw std::runtime_error("only the CC metric is supported, got '" + m.name + "'");
  if (m.params.size() < 2) throw std::runtime_error("CC[fixed,moving,weight,radius] needs the two images");

  synx_params p;
  synx_params_default(&p, dim);
  if (t.params.empty()) throw std::runtime_error("SyN[gradientStep,...] needs a gradient step");
  p.learning_rate = std::atof(t.params[0].c_str());
  if (t.params.size() > 1) p.update_variance = std::atof(t.params[1].c_str());
  if (t.params.size() > 2) p.total_variance = std::atof(t.params[2].c_str());
  if (m.params.size() > 3) p.cc_radius = std::atoi(m.params[3].c_str());
  // -c [iterations,threshold,window]
  OptionCall c = parse_call(one("convergence", ""));
  std::vector<int> iters;
  if (!c.params.empty()) {
    iters = parse_x_vector<int>(c.params[0]);
    if (c.params.size() > 1) p.convergence_threshold = std::atof(c.params[1].c_str());
    if (c.params.size() > 2) p.convergence_window = std::atoi(c.params[2].c_str());
  } else if (!c.name.empty()) {
    iters = parse_x_vector<int>(c.name);
  }
  if (iters.empty()) throw std::runtime_error("no convergence criteria (-c) were given");
  const int L = (int)iters.size();
  if (L > SYNX_MAX_LEVELS) throw std::runtime_error("at most 8 levels are supported");
  std::vector<int> shrink = parse_x_vector<int>(one("shrink-factors", ""));
  std::string sig = one("smoothing-sigmas", "");
  if (sig.find("mm") != std::string::npos) {
    p.sigmas_in_mm = 1;
    sig.replace(sig.find("mm"), 2, "");
  } else if (sig.find("vox") != std::string::npos) {
    sig.replace(sig.find("vox"), 3, "");
  }
  std::vector<double> sigmas = parse_x_vector<double>(sig);
  if (sigmas.size() == 1) sigmas.resize(L, sigmas[0]);
  if ((int)shrink.size() != L || (int)sigmas.size() != L)
    throw std::runtime_error("the number of shrink factors and smoothing sigmas must match the levels of -c");
  p.n_levels = L;
  for (int l = 0; l < L; ++l) {
    p.iterations[l] = iters[l];
    p.shrink_factors[l] = shrink[l];
    p.smoothing_sigmas[l] = sigmas[l];
  }
  // the moving image matched to the fixed one after the window (PreprocessImage,
  // Examples/itkantsRegistrationHelper.hxx:1135-1143)
  p.histogram_match = histogram_matching ? 1 : 0;
  if (opt.count("winsorize-image-intensities")) {
    OptionCall w = parse_call(one("winsorize-image-intensities", ""));
    if (w.params.size() > 0) p.winsor_lower = (float)std::atof(w.params[0].c_str());
    if (w.params.size() > 1) p.winsor_upper = (float)std::atof(w.params[1].c_str());
  }
  OptionCall o = parse_call(one("output", ""));
  std::string prefix = o.params.empty() ? o.name : o.params[0];
  if (prefix.empty()) throw std::runtime_error("no output prefix (-o) was given");
  const std::string warped = o.params.size() > 1 ? o.params[1] : "";
  const std::string inv_warped = o.params.size() > 2 ? o.params[2] : "";

  nifti::Image fixed = nifti::read(m.params[0]);
  nifti::Image moving = nifti::read(m.params[1]);
  if (fixed.components != 1 || moving.components != 1) throw std::runtime_error("scalar images expected");
  synx_geom gf = to_geom(fixed, dim), gm = to_geom(moving, dim);
  // the initial transform folded into the moving image's geometry: its voxel i is placed at
  // Init^-1(p_i), so sampling it at q reads the moving image at Init(q)
  if (!init.empty()) gm = push_forward(gm, init_inverse);
  if (verbose) {
    out << "  Stage 0: SyN[" << p.learning_rate << "," << p.update_variance << "," << p.total_variance
        << "], CC[radius " << p.cc_radius << "], " << L << " levels on GPU " << gpu << std::endl;
    if (!init.empty())
      out << "  initial moving transform: " << init.size()
          << " linear transform(s), folded into the moving image geometry" << std::endl;
  }
  // -x [fixedMask,movingMask] or -x fixedMask (antsRegistrationTemplateHeader.h:363-425): a file that
  // does not exist (NULL, for instance) means no mask for that image; one stage, so one -x
  nifti::Image mask_f, mask_m;
  bool have_mask_f = false, have_mask_m = false;
  if (opt.count("masks")) {
    if (opt["masks"].size() != 1) throw std::runtime_error("one --masks option per stage: this is one stage");
    OptionCall x = parse_call(opt["masks"][0]);
    std::vector<std::string> names = x.params.empty() ? std::vector<std::string>{x.name} : x.params;
    auto exists = [](const std::string& f) {
      FILE* fh = std::fopen(f.c_str(), "rb");
      if (fh) std::fclose(fh);
      return fh != nullptr;
    };
    if (!names.empty() && exists(names[0])) {
      mask_f = nifti::read(names[0]);
      have_mask_f = true;
    }
    if (names.size() > 1 && exists(names[1])) {
      mask_m = nifti::read(names[1]);
      have_mask_m = true;
    }
    if ((have_mask_f && mask_f.components != 1) || (have_mask_m && mask_m.components != 1))
      throw std::runtime_error("scalar mask images expected");
  }
  synx_ctx* ctx = nullptr;
  if (synx_create(&p, gpu, nullptr, &ctx) != 0) throw std::runtime_error(std::string("synx_create: ") + synx_last_error(nullptr));
  struct Guard {
    synx_ctx* c;
    ~Guard() { synx_destroy(c); }
  } guard{ctx};
  if (have_mask_f || have_mask_m) {
    const synx_geom gmf = have_mask_f ? to_geom(mask_f, dim) : synx_geom{};
    // the moving mask is sampled through the same transforms as the moving image
    synx_geom gmm = have_mask_m ? to_geom(mask_m, dim) : synx_geom{};
    if (have_mask_m && !init.empty()) gmm = push_forward(gmm, init_inverse);
    if (synx_set_masks(ctx, have_mask_f ? mask_f.data.data() : nullptr, have_mask_f ? &gmf : nullptr,
                       have_mask_m ? mask_m.data.data() : nullptr, have_mask_m ? &gmm : nullptr) != 0)
      throw std::runtime_error(std::string("synx_set_masks: ") + synx_last_error(ctx));
    if (verbose)
      out << "  metric masks: fixed " << (have_mask_f ? "yes" : "no") << ", moving " << (have_mask_m ? "yes" : "no")
          << std::endl;
  }
  auto t0 = std::chrono::steady_clock::now();
  if (synx_set_images(ctx, fixed.data.data(), &gf, moving.data.data(), &gm) != 0)
    throw std::runtime_error(std::string("synx_set_images: ") + synx_last_error(ctx));
  if (!state_fields.empty()) {
    // the SyN stage starts from the restored fixed-to-middle and moving-to-middle fields
    // (itkantsRegistrationHelper.hxx:2093-2125)
    const synx_geom gs = composite::field_geom(state_fields[0], dim);
    for (int k = 1; k < 4; ++k) {
      composite::field_geom(state_fields[k], dim);
      if (state_fields[k].fixed != state_fields[0].fixed)
        throw std::runtime_error("--restore-state: the four SyN fields do not share one grid");
    }
    if (synx_set_initial_half_fields(ctx, state_fields[0].field.data(), state_fields[1].field.data(),
                                     state_fields[2].field.data(), state_fields[3].field.data(), &gs) != 0)
      throw std::runtime_error(std::string("synx_set_initial_half_fields: ") + synx_last_error(ctx));
    if (verbose) out << "  SyN stage initialized from the restored registration state" << std::endl;
  }
  int64_t printed = 0;
  for (int l = 0; l < L; ++l) {
    auto tl = std::chrono::steady_clock::now();
    if (synx_run_level(ctx, l) != 0) throw std::runtime_error(std::string("synx_run_level: ") + synx_last_error(ctx));
    const double level_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - tl).count();
    if (verbose) {
      int64_t n = 0;
      synx_get_log(ctx, nullptr, nullptr, nullptr, nullptr, nullptr, 0, &n);
      std::vector<int32_t> lv(n), it(n), ki(n);
      std::vector<double> me(n), cv(n);
      synx_get_log(ctx, lv.data(), it.data(), me.data(), cv.data(), ki.data(), n, &n);
      const double t_level0 = std::chrono::duration<double>(tl - t0).count();
      const int64_t k_level = n - printed;
      out << "  Current level = " << l + 1 << " of " << L << "\n    number of iterations = " << iters[l]
          << "\n    shrink factors = " << shrink[l] << "\n    smoothing sigmas = " << sigmas[l]
          << (p.sigmas_in_mm ? " mm" : " vox") << "\n";
      out << "XXDIAGNOSTIC,Iteration,metricValue,convergenceValue,ITERATION_TIME_INDEX,SINCE_LAST\n";
      for (int64_t k = printed; k < n; ++k) {
        const double dt = level_s / std::max<int64_t>(k_level, 1);
        out << " 1DIAGNOSTIC, " << std::setw(5) << it[k] << ", " << std::scientific << std::setprecision(12)
            << me[k] << ", " << std::setprecision(12) << cv[k] << ", " << std::setprecision(4)
            << t_level0 + dt * (double)(k - printed + 1) << ", " << std::setprecision(4) << dt << ", " << std::endl;
        out.unsetf(std::ios::scientific);
      }
      printed = n;
    }
  }
  synx_geom go;
  synx_get_output_geom(ctx, &go);
  const long long No = go.size[0] * go.size[1] * go.size[2];
  std::vector<float> fwd((size_t)No * dim), inv((size_t)No * dim);
  if (synx_get_fields(ctx, fwd.data(), inv.data()) != 0)
    throw std::runtime_error(std::string("synx_get_fields: ") + synx_last_error(ctx));
  // output files in the precision the reference writes them: float with --float 1, double by default
  // (antsRegistration.cxx:488-491); the values are computed in float either way
  const int out_type = use_float ? 16 : 64;
  auto typed = [out_type](nifti::Image im) {
    im.out_datatype = out_type;
    return im;
  };
  // the initial transforms in composite order (the one acting last first), collapsed to one affine
  // transform when the output transforms are collapsed
  std::vector<synx_linear> queue;
  for (auto it = init.rbegin(); it != init.rend(); ++it) queue.push_back(it->linear);
  std::vector<synx_linear> out_queue = queue;
  if (collapse && !init.empty()) out_queue.assign(1, linear_of(init_map, dim, init_center));
  if (!save_state.empty()) {
    // the registration state (antsRegistrationTemplateHeader.h:1307-1346): the initial transforms,
    // then fixed-to-middle, its inverse, moving-to-middle, its inverse
    std::vector<float> hf[4];
    for (auto& h : hf) h.resize((size_t)No * dim);
    if (synx_get_half_fields(ctx, hf[0].data(), hf[1].data(), hf[2].data(), hf[3].data()) != 0)
      throw std::runtime_error(std::string("synx_get_half_fields: ") + synx_last_error(ctx));
    std::vector<composite::Item> items;
    for (const synx_linear& t : queue) items.push_back(composite::linear_item(t, dim));
    for (const auto& h : hf) items.push_back(composite::field_item(go, h, !use_float));
    composite::write(save_state, dim, items);
  }
  if (composite_out) {
    // prefixComposite and prefixInverseComposite (antsRegistrationTemplateHeader.h:1394-1424): the
    // initial transforms then the SyN field; the inverse lists the inverses in reverse order
    std::vector<composite::Item> fw, iv;
    for (const synx_linear& t : out_queue) fw.push_back(composite::linear_item(t, dim));
    fw.push_back(composite::field_item(go, fwd, !use_float));
    iv.push_back(composite::field_item(go, inv, !use_float));
    for (auto it = out_queue.rbegin(); it != out_queue.rend(); ++it) {
      Map mi;
      if (!inverse(map_of(*it, false), mi)) throw std::runtime_error("an initial transform is singular");
      iv.push_back(composite::linear_item(linear_of(mi, dim, it->center), dim));
    }
    composite::write(prefix + "Composite.txt", dim, fw);
    composite::write(prefix + "InverseComposite.txt", dim, iv);
  }
  // file names as antsRegistrationTemplateHeader.h:1436-1458 numbers them: with initial transforms
  // and collapsing, prefix0GenericAffine.mat holds them and the SyN fields are transform 1; without
  // collapsing the initial transforms are not rewritten and the SyN fields follow them, except those
  // a restored state brought, which are written one by one (the numbering starts after the -r
  // options, :1434, and a restored state has none)
  int warp_index = 0;
  if (!composite_out && !init.empty()) {
    warp_index = collapse ? 1 : (restore_state.empty() ? n_init : (int)queue.size());
    if (!collapse && !restore_state.empty()) {
      for (size_t k = 0; k < queue.size(); ++k) {
        const std::string name = prefix + std::to_string(k) + "GenericAffine.mat";
        if (synx_write_linear_transform(name.c_str(), &queue[k]) != 0)
          throw std::runtime_error(std::string("synx_write_linear_transform: ") + synx_last_error(nullptr));
      }
    } else if (collapse) {
      const synx_linear total = linear_of(init_map, dim, init_center);
      if (synx_write_linear_transform((prefix + "0GenericAffine.mat").c_str(), &total) != 0)
        throw std::runtime_error(std::string("synx_write_linear_transform: ") + synx_last_error(nullptr));
    } else {
      // derived initial transforms are written out when they are not collapsed (:229-250)
      for (const auto& d : derived) {
        const std::string name = prefix + std::to_string(d.first) + "DerivedInitialMovingTranslation.mat";
        if (synx_write_linear_transform(name.c_str(), &d.second) != 0)
          throw std::runtime_error(std::string("synx_write_linear_transform: ") + synx_last_error(nullptr));
      }
    }
  }
  const std::string wi = std::to_string(warp_index);
  if (!composite_out) {
    nifti::write(prefix + wi + "Warp.nii.gz", typed(field_image(go, fwd)));
    nifti::write(prefix + wi + "InverseWarp.nii.gz", typed(field_image(go, inv)));
  }
  if (!warped.empty()) nifti::write(warped, typed(like(fixed, warp_on_device(moving, gm, fwd, go))));
  if (!inv_warped.empty()) {
    std::vector<float> inv_on_moving = resample_on_device(inv, go, gm);
    nifti::write(inv_warped, typed(like(moving, warp_on_device(fixed, gf, inv_on_moving, gm))));
  }
  if (verbose) {
    const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    out << "  Elapsed time (stage 0): " << total << std::endl;
  }
  return EXIT_SUCCESS;
}

}  // namespace

int antsRegistration(std::vector<std::string> args, std::ostream* out) {
  std::ostream& os = out ? *out : std::cout;
  try {
    return run(args, os);
  } catch (const std::exception& e) {
    std::cerr << "antsRegistrationSyN_b200: " << e.what() << std::endl;
    return EXIT_FAILURE;
  }
}

}  // namespace ants_b200

namespace ants {

int antsRegistration(std::vector<std::string> args, std::ostream* out_stream) {
  return ants_b200::antsRegistration(std::move(args), out_stream);
}

}  // namespace ants

#ifndef SYNX_CLI_NO_MAIN
int main(int argc, char** argv) {
  std::vector<std::string> args(argv + 1, argv + argc);
  return ants::antsRegistration(args, &std::cout);
}
#endif
