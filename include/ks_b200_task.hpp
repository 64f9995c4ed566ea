/* keepsake-b200: the TOML task boundary, for C++ hosts.
 *
 * Mirrors keepsake's configuration service (config.h:17-140) for the small_pt path: a TOML
 * document with asset tables ([bsdf.NAME], [material.NAME], [mesh_asset.NAME]) and an array of
 * tasks ([[task]] with `type`, optional `task_dir` and `override`), run in order, each in its own
 * output directory (ConfigServiceInternal::run_all_tasks, config.cpp:262-312).  Tasks are
 * functions with keepsake's ConfigTask signature (config.h:119).  Registered:
 *   "small_pt" and "small_pt_b200": small_pt (small_pt.cpp:180-300) on the GPU through the C ABI,
 *   reading the same keys (object or compound_object, material, sky, light (point,
 *   directional), pixel_filter (box, gaussian, blackman_harris), backdrop, bounces, clamp_direct,
 *   clamp_indirect, render_width, render_height, crop_*, spp, scale_ray_diff, rng_seed,
 *   spp_prog_interval, camera or camera_animation with camera_animation_offset / _count) plus
 *   the `emission` key of a material.  After every spp interval the composited image is written
 *   to TASK_DIR/small_pt_spp<N>[_<frame>].exr (OpenEXR, FP32 RGB; ZIP
 *   compression where the reference's tinyexr call asks for PIZ: both lossless).  Sky maps are
 *   read from .exr, .hdr (and .pfm) files.
 *   "convert_mesh_asset": each mesh asset of `assets` written to TASK_DIR/<name>.bin in keepsake's
 *   binary mesh asset format (mesh_asset.cpp:180-240, 301-311).
 * Mesh assets: `path` + `format` "obj" (twosided, default false; use_smooth_normal, default true;
 * positions, texcoords and normals) or "bin", with an optional `to_world` transform
 * (create_mesh_asset, mesh_asset.cpp:243-266).  Compound mesh assets
 * ([compound_mesh_asset.NAME], the task's `compound_object`): a glTF 2.0 file (`format` "glb" or
 * "gltf"; `load_materials` for its constant metallic-roughness materials), prototypes per glTF
 * mesh and instances per node (create_compound_mesh_asset, mesh_asset.cpp:1114-1132).
 * Errors throw std::runtime_error (the reference asserts); the C entry point ks_config_run in
 * ks_b200.h returns a status instead.
 */
#pragma once
#include <filesystem>
#include <functional>
#include <memory>
#include <string>
#include <string_view>

namespace ks_b200
{

struct ConfigArgsInternal;

// A view of one node of the configuration (ConfigArgs, config.h:17-90).
struct ConfigArgs
{
    explicit ConfigArgs(std::shared_ptr<ConfigArgsInternal> internal);
    ConfigArgs operator[](std::string_view key) const;
    ConfigArgs operator[](int index) const;
    bool contains(std::string_view key) const;
    int array_size() const;
    int load_integer(std::string_view key) const;
    int load_integer(std::string_view key, int default_value) const;
    float load_float(std::string_view key) const;
    float load_float(std::string_view key, float default_value) const;
    bool load_bool(std::string_view key) const;
    bool load_bool(std::string_view key, bool default_value) const;
    std::string load_string(std::string_view key) const;
    std::string load_string(std::string_view key, std::string_view default_value) const;
    std::string load_string(int index) const;
    void load_vec3(std::string_view key, float out[3]) const;
    // Transform field (config.cpp:204-260): matrix_rm | matrix_cm | scale + rotation{euler|quat}
    // + translation; row-major 4x4 out.
    void load_transform(std::string_view key, float out[16]) const;
    std::filesystem::path load_path(std::string_view key) const; // relative to the asset root

    std::shared_ptr<ConfigArgsInternal> internal;
};

// keepsake's ConfigTask (config.h:119): (task arguments, task output directory, task index).
using ConfigTask = std::function<void(const ConfigArgs &args, const std::filesystem::path &task_dir, int task_id)>;

// The GPU small_pt task.  Device: KS_B200_DEVICE environment variable, else 0.
void small_pt_b200(const ConfigArgs &args, const std::filesystem::path &task_dir, int task_id);
void convert_mesh_asset(const ConfigArgs &args, const std::filesystem::path &task_dir, int task_id);

struct ConfigServiceImpl;

// ConfigService (config.h:121-140) with the small_pt tasks registered.
class ConfigService
{
  public:
    ConfigService();
    ~ConfigService();
    void parse_file(const std::filesystem::path &file_path);
    void parse(std::string_view text);
    void set_asset_root_dir(const std::filesystem::path &root);
    void set_output_directory(const std::filesystem::path &dir);
    void register_task(std::string_view name, const ConfigTask &task);
    std::filesystem::path output_directory() const;
    void run_all_tasks() const;

  private:
    std::unique_ptr<ConfigServiceImpl> impl;
};

} // namespace ks_b200
