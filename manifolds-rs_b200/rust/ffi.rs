//! umapcu: the B200 (sm_100a) CUDA backend of manifolds-rs's `"adam_gpu"`
//! optimiser slot and of its UMAP graph stage.
//!
//! UNCOMPILED: no Rust toolchain (cargo / rustc) exists where this library is
//! built and tested, so this file has never been through rustc. It is the
//! binding a manifolds-rs maintainer adds as `src/training/umapcu_ffi.rs`,
//! written against manifolds-rs 0.3.15's types:
//!
//! * `UmapOptimParams<f32>` (src/training/umap_optimisers.rs:24-45),
//! * `DensState<f32>` / `DensParams<f32>` (src/utils/density.rs:69-79,
//!   :140-160),
//! * `CoordinateList<f32>` (src/data/structures.rs:22-59),
//! * `ManifoldsError` (src/errors.rs:7-118), plus one variant this binding
//!   needs (below).
//!
//! It links `libumapcu.so` (build.rs: `cargo:rustc-link-search=native=<dir>`,
//! `cargo:rustc-link-lib=dylib=umapcu`) and calls the C ABI of
//! `include/umapcu.h`. Entry points:
//!
//! * [`optimise_embedding_adam_cuda`] replaces `optimise_embedding_adam_gpu`
//!   (src/training/umap_optimiser_gpu.rs:1302-1310; the generic runtime and
//!   its `device` argument are dropped) in the `UmapOptimiserGpu::AdamGpu` arm
//!   of `umap_gpu_inner` (src/lib.rs:3657-3690);
//! * [`construct_umap_graph_cuda`] replaces the smooth_knn_dist ->
//!   knn_to_coo -> symmetrise_graph -> filter_weak_edges chain of
//!   `construct_umap_graph_gpu` (src/lib.rs:3421-3431);
//! * [`dens_state_new_cuda`] replaces `DensState::new`
//!   (src/utils/density.rs:181-201).
//!
//! Errors. Statuses 1-3 are the crate's own `NoData`, `NoGraphEdges` and
//! `DegenerateLocalRadii`. The device-side statuses keep their identity in
//! [`UmapcuError`]; `ManifoldsError::CubeclUtilsError` wraps an error type of
//! another crate (`cubecl_utils_rs::CubeclUtilsErrors`, src/errors.rs:54) that
//! this binding cannot construct, so the maintainer adds to `ManifoldsError`:
//!
//! ```ignore
//! /// Errors of the umapcu CUDA backend
//! #[error("umapcu CUDA backend: {0}")]
//! Umapcu(#[from] crate::training::umapcu_ffi::UmapcuError),
//! ```

use std::os::raw::{c_char, c_int};

use thiserror::Error;

use crate::data::structures::CoordinateList;
use crate::errors::ManifoldsError;
use crate::training::umap_optimisers::UmapOptimParams;
use crate::utils::density::DensState;

// ------------------------------------------------------------------ C ABI

/// `umapcu_optim_params` (include/umapcu.h).
#[repr(C)]
struct OptimParams {
    a: f32,
    b: f32,
    lr: f32,
    gamma: f32,
    n_epochs: u32,
    neg_sample_rate: u32,
    min_dist: f32,
    beta1: f32,
    beta2: f32,
    eps: f32,
}

/// `umapcu_graph_params` (include/umapcu.h).
#[repr(C)]
struct GraphParams {
    bandwidth: f32,
    local_connectivity: f32,
    mix_weight: f32,
}

/// `umapcu_dens` (include/umapcu.h); `r` / `mu_sum` borrow the state's
/// vectors for the duration of the call.
#[repr(C)]
struct Dens {
    lambda: f32,
    frac: f32,
    var_shift: f32,
    r: *const f32,
    mu_sum: *const f32,
    mu_tot: f32,
}

const OPT_ADAM: u32 = 0;
const NEG_REF_HASH: u32 = 0;

#[link(name = "umapcu")]
extern "C" {
    fn umapcu_status_string(status: c_int) -> *const c_char;
    fn umapcu_optimise_embedding(
        embd: *mut f32,
        n: u32,
        n_dim: u32,
        adj_ptr: *const u64,
        adj_col: *const u32,
        adj_w: *const f32,
        params: *const OptimParams,
        dens: *const Dens,
        seed: u64,
        optimiser: u32,
        sampler: u32,
        verbose: c_int,
    ) -> c_int;
    fn umapcu_construct_umap_graph(
        knn_idx: *const i32,
        knn_dist: *const f32,
        n: u32,
        k: u32,
        params: *const GraphParams,
        n_epochs: u32,
        capacity: u64,
        row: *mut u32,
        col: *mut u32,
        val: *mut f32,
        nnz: *mut u64,
        sigma: *mut f32,
        rho: *mut f32,
    ) -> c_int;
    fn umapcu_dens_state_new(
        n: u32,
        nnz: u64,
        row: *const u32,
        col: *const u32,
        val: *const f32,
        knn_idx: *const i32,
        knn_dist: *const f32,
        k: u32,
        distances_squared: c_int,
        r: *mut f32,
        mu_sum: *mut f32,
        mu_tot: *mut f32,
    ) -> c_int;
}

// ------------------------------------------------------------------ errors

/// The umapcu statuses that have no `ManifoldsError` variant of their own
/// (include/umapcu.h `umapcu_status`, values 4-10).
#[derive(Debug, Error, Clone, Copy, PartialEq, Eq)]
pub enum UmapcuError {
    /// Device memory allocation failed (4).
    #[error("CUDA allocation failed")]
    CudaAlloc,
    /// A launch or runtime call failed (5).
    #[error("CUDA launch or runtime error")]
    CudaLaunch,
    /// A bounded device wait gave up (6).
    #[error("bounded device wait timed out")]
    Timeout,
    /// An argument was rejected before any device work (7).
    #[error("bad argument")]
    BadArg,
    /// No usable CUDA device (8).
    #[error("no CUDA device")]
    NoDevice,
    /// An output capacity, device budget or scratch size was exceeded (9).
    #[error("capacity exceeded")]
    Capacity,
    /// A served job was cancelled or its server shut down (10).
    #[error("cancelled")]
    Cancelled,
    /// A status this binding does not know (a newer library).
    #[error("unknown umapcu status {0}")]
    Unknown(i32),
}

/// Maps a `umapcu_status` onto the crate's error type, one variant per
/// status.
fn status(rc: c_int) -> Result<(), ManifoldsError> {
    let e = match rc {
        0 => return Ok(()),
        1 => return Err(ManifoldsError::NoData),
        2 => return Err(ManifoldsError::NoGraphEdges),
        3 => return Err(ManifoldsError::DegenerateLocalRadii),
        4 => UmapcuError::CudaAlloc,
        5 => UmapcuError::CudaLaunch,
        6 => UmapcuError::Timeout,
        7 => UmapcuError::BadArg,
        8 => UmapcuError::NoDevice,
        9 => UmapcuError::Capacity,
        10 => UmapcuError::Cancelled,
        other => UmapcuError::Unknown(other),
    };
    Err(ManifoldsError::Umapcu(e))
}

/// The library's own text for a status (static storage).
pub fn status_text(rc: i32) -> String {
    unsafe {
        let p = umapcu_status_string(rc as c_int);
        if p.is_null() {
            return String::new();
        }
        std::ffi::CStr::from_ptr(p).to_string_lossy().into_owned()
    }
}

fn optim_params(p: &UmapOptimParams<f32>) -> Result<OptimParams, ManifoldsError> {
    let n_epochs = u32::try_from(p.n_epochs).map_err(|_| ManifoldsError::Umapcu(UmapcuError::BadArg))?;
    let neg = u32::try_from(p.neg_sample_rate).map_err(|_| ManifoldsError::Umapcu(UmapcuError::BadArg))?;
    Ok(OptimParams {
        a: p.a,
        b: p.b,
        lr: p.lr,
        gamma: p.gamma,
        n_epochs,
        neg_sample_rate: neg,
        min_dist: p.min_dist,
        beta1: p.beta1,
        beta2: p.beta2,
        eps: p.eps,
    })
}

fn to_u32(x: usize) -> Result<u32, ManifoldsError> {
    u32::try_from(x).map_err(|_| ManifoldsError::Umapcu(UmapcuError::BadArg))
}

// ------------------------------------------------------------ entry points

/// Drop-in for `optimise_embedding_adam_gpu` (src/training/
/// umap_optimiser_gpu.rs:1302-1310) on the CUDA backend: the same arguments
/// without the runtime's `device`, the same in-place update of `embd`, the
/// same errors for empty data and edgeless graphs. The reference's own
/// negative-sample hash (`gpu_hash_neg`, :611-624) is used, so the run draws
/// the reference's negatives.
pub fn optimise_embedding_adam_cuda(
    embd: &mut [Vec<f32>],
    graph: &[Vec<(usize, f32)>],
    params: &UmapOptimParams<f32>,
    dens: Option<&DensState<f32>>,
    seed: u64,
    verbose: usize,
) -> Result<(), ManifoldsError> {
    let n = embd.len();
    if n == 0 {
        return Err(ManifoldsError::NoData);
    }
    let n_dim = embd[0].len();
    if embd.iter().any(|p| p.len() != n_dim) || graph.len() != n {
        return Err(ManifoldsError::Umapcu(UmapcuError::BadArg));
    }
    let mut flat: Vec<f32> = Vec::with_capacity(n * n_dim);
    for p in embd.iter() {
        flat.extend_from_slice(p);
    }
    let nnz: usize = graph.iter().map(|r| r.len()).sum();
    let mut ptr: Vec<u64> = Vec::with_capacity(n + 1);
    let mut col: Vec<u32> = Vec::with_capacity(nnz);
    let mut w: Vec<f32> = Vec::with_capacity(nnz);
    ptr.push(0);
    for row in graph {
        for &(j, x) in row {
            if j >= n {
                return Err(ManifoldsError::Umapcu(UmapcuError::BadArg));
            }
            col.push(j as u32);
            w.push(x);
        }
        ptr.push(col.len() as u64);
    }
    let p = optim_params(params)?;
    let d = dens.map(|s| Dens {
        lambda: s.params.lambda,
        frac: s.params.frac,
        var_shift: s.params.var_shift,
        r: s.r.as_ptr(),
        mu_sum: s.mu_sum.as_ptr(),
        mu_tot: s.mu_tot,
    });
    let dp = d.as_ref().map_or(std::ptr::null(), |x| x as *const Dens);
    status(unsafe {
        umapcu_optimise_embedding(
            flat.as_mut_ptr(),
            to_u32(n)?,
            to_u32(n_dim)?,
            ptr.as_ptr(),
            col.as_ptr(),
            w.as_ptr(),
            &p,
            dp,
            seed,
            OPT_ADAM,
            NEG_REF_HASH,
            verbose.min(i32::MAX as usize) as c_int,
        )
    })?;
    for (i, point) in embd.iter_mut().enumerate() {
        point.copy_from_slice(&flat[i * n_dim..(i + 1) * n_dim]);
    }
    Ok(())
}

/// The graph stage of `construct_umap_graph_gpu` (src/lib.rs:3421-3431) on
/// the CUDA backend: kNN lists (self excluded, squared Euclidean distances
/// as the ANN backends return them) -> the symmetrised, filtered fuzzy
/// graph, rows grouped and columns ascending as `symmetrise_csr` returns it.
pub fn construct_umap_graph_cuda(
    knn_indices: &[Vec<usize>],
    knn_dists: &[Vec<f32>],
    bandwidth: f32,
    local_connectivity: f32,
    mix_weight: f32,
    n_epochs: usize,
) -> Result<CoordinateList<f32>, ManifoldsError> {
    let n = knn_indices.len();
    if n == 0 {
        return Err(ManifoldsError::NoData);
    }
    let k = knn_indices[0].len();
    if knn_dists.len() != n
        || knn_indices.iter().any(|r| r.len() != k)
        || knn_dists.iter().any(|r| r.len() != k)
    {
        return Err(ManifoldsError::Umapcu(UmapcuError::BadArg));
    }
    let mut idx: Vec<i32> = Vec::with_capacity(n * k);
    for r in knn_indices {
        for &j in r {
            idx.push(i32::try_from(j).map_err(|_| ManifoldsError::Umapcu(UmapcuError::BadArg))?);
        }
    }
    let dist: Vec<f32> = knn_dists.iter().flatten().copied().collect();
    let cap = 2 * n * k;
    let (mut row, mut col, mut val) = (vec![0u32; cap], vec![0u32; cap], vec![0f32; cap]);
    let mut nnz: u64 = 0;
    let gp = GraphParams {
        bandwidth,
        local_connectivity,
        mix_weight,
    };
    status(unsafe {
        umapcu_construct_umap_graph(
            idx.as_ptr(),
            dist.as_ptr(),
            to_u32(n)?,
            to_u32(k)?,
            &gp,
            to_u32(n_epochs)?,
            cap as u64,
            row.as_mut_ptr(),
            col.as_mut_ptr(),
            val.as_mut_ptr(),
            &mut nnz,
            std::ptr::null_mut(),
            std::ptr::null_mut(),
        )
    })?;
    let m = nnz as usize;
    Ok(CoordinateList {
        row_indices: row[..m].iter().map(|&x| x as usize).collect(),
        col_indices: col[..m].iter().map(|&x| x as usize).collect(),
        values: val[..m].to_vec(),
        n_samples: n,
    })
}

/// `DensState::new` (src/utils/density.rs:181-201) on the CUDA backend, for
/// the symmetrised graph and the kNN lists it came from.
pub fn dens_state_new_cuda(
    params: crate::utils::density::DensParams<f32>,
    graph: &CoordinateList<f32>,
    knn_indices: &[Vec<usize>],
    knn_dists: &[Vec<f32>],
    distances_squared: bool,
) -> Result<DensState<f32>, ManifoldsError> {
    let n = graph.n_samples;
    if n == 0 || knn_indices.len() != n {
        return Err(ManifoldsError::NoData);
    }
    let k = knn_indices[0].len();
    let row: Vec<u32> = graph.row_indices.iter().map(|&x| x as u32).collect();
    let col: Vec<u32> = graph.col_indices.iter().map(|&x| x as u32).collect();
    let mut idx: Vec<i32> = Vec::with_capacity(n * k);
    for r in knn_indices {
        for &j in r {
            idx.push(i32::try_from(j).map_err(|_| ManifoldsError::Umapcu(UmapcuError::BadArg))?);
        }
    }
    let dist: Vec<f32> = knn_dists.iter().flatten().copied().collect();
    let (mut r, mut mu_sum, mut mu_tot) = (vec![0f32; n], vec![0f32; n], 0f32);
    status(unsafe {
        umapcu_dens_state_new(
            to_u32(n)?,
            row.len() as u64,
            row.as_ptr(),
            col.as_ptr(),
            graph.values.as_ptr(),
            idx.as_ptr(),
            dist.as_ptr(),
            to_u32(k)?,
            distances_squared as c_int,
            r.as_mut_ptr(),
            mu_sum.as_mut_ptr(),
            &mut mu_tot,
        )
    })?;
    Ok(DensState {
        params,
        r,
        mu_sum,
        mu_tot,
    })
}
