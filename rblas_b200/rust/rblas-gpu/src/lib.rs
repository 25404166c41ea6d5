//! # rblas-gpu — rblas's Level-3 API on a B200
//!
//! Drop-in twins of `rblas::level3` and `rblas::complex3` whose arithmetic runs
//! in librblas_b200.so (hand-written sm_100a kernels) behind its C ABI
//! (`include/rblas_b200.h`). Arguments, validation order and errors are
//! rblas's: `try_gemm` returns the same `BlasError` for the same bad
//! arguments (`src/level3.rs:68-140`), and `gemm` panics where rblas panics
//! (it is `try_gemm(..).unwrap()`).
//!
//! The GPU adds failure modes rblas does not have (a CUDA call failing, a
//! device allocation failing, a bounded device wait giving up). The
//! rblas-shaped functions panic on those, since `BlasError` has no variant
//! for them; [`level3::try_gemm_prec`], [`complex3::try_gemm_prec`] and
//! [`level3::dgemm_dev`] return them as [`Error::Device`].
//!
//! Beside the drop-in (the plain form: true FP32 / FP64 products) the
//! precision forms are reachable through [`level3::try_gemm_prec`]: 3xBF16 /
//! BF16X6 for f32 and Ozaki INT8-slice emulation for f64.
//!
//! [`level1`], [`level2`], [`complex1`] and [`complex2`] are the same for
//! rblas's vector and matrix-vector routines; like rblas's, they panic on
//! arguments they cannot use.

use core::fmt;
use std::os::raw::c_void;

pub use rblas::{BlasError, Complex, Diag, Layout, Side, Transpose, Uplo, C32, C64};

/// Arithmetic form of a GEMM call (`rb_precision`).
#[derive(Copy, Clone, Debug, PartialEq, Eq)]
pub enum Precision {
    /// The drop-in: true FP32 / FP64 products.
    Plain = 0,
    /// f32: hi*hi + hi*lo + lo*hi of a bf16 hi/lo split on the tensor cores.
    Bf16x3 = 1,
    /// f64: INT8 slices with per-row/column power-of-two scaling, exact INT32 products.
    Ozaki = 2,
    /// f32: the six products of weight <= 2 of a three-plane bf16 split.
    Bf16x6 = 3,
}

/// A failed call: an rblas argument error, or a failure on the GPU side.
#[derive(Clone, Debug, PartialEq, Eq)]
pub enum Error {
    /// The same error rblas's `try_*` function returns for these arguments.
    Blas(BlasError),
    /// A status rblas has no counterpart for (`rb_status` code, the CUDA
    /// error code where there is one, the device error word or other detail).
    Device { code: i32, cuda_error: i32, detail: u64 },
}

impl fmt::Display for Error {
    fn fmt(&self, f: &mut fmt::Formatter<'_>) -> fmt::Result {
        match self {
            Error::Blas(e) => write!(f, "{e}"),
            Error::Device { code, cuda_error, detail } => {
                let s = unsafe { std::ffi::CStr::from_ptr(ffi::rb_status_string(*code)) };
                write!(f, "rblas-gpu: {} (status {code}, cuda {cuda_error}, detail {detail:#x})", s.to_string_lossy())
            }
        }
    }
}

impl std::error::Error for Error {}

/// The raw C ABI (`include/rblas_b200.h`).
pub mod ffi {
    use super::*;

    #[repr(C)]
    #[derive(Copy, Clone, Debug, Default)]
    pub struct RbError {
        pub code: i32,
        pub which: u8,
        pub got: u64,
        pub min_or_need: u64,
        pub cuda_error: i32,
    }

    extern "C" {
        pub fn rb_status_string(status: i32) -> *const std::os::raw::c_char;
        // level3::try_gemm (src/level3.rs:68-103), host slices + lengths
        pub fn rb_sgemm_prec(layout: i32, transa: i32, transb: i32, m: usize, n: usize, k: usize, alpha: f32,
                             a: *const f32, lda: usize, a_len: usize, b: *const f32, ldb: usize, b_len: usize,
                             beta: f32, c: *mut f32, ldc: usize, c_len: usize, prec: i32, err: *mut RbError) -> i32;
        pub fn rb_dgemm_prec(layout: i32, transa: i32, transb: i32, m: usize, n: usize, k: usize, alpha: f64,
                             a: *const f64, lda: usize, a_len: usize, b: *const f64, ldb: usize, b_len: usize,
                             beta: f64, c: *mut f64, ldc: usize, c_len: usize, prec: i32, err: *mut RbError) -> i32;
        // complex3::gemm (src/complex3.rs:27-74); Complex<T> is #[repr(C)] {re, im}
        pub fn rb_cgemm(transa: i32, transb: i32, m: usize, n: usize, k: usize, alpha: C32, a: *const C32,
                        lda: usize, a_len: usize, b: *const C32, ldb: usize, b_len: usize, beta: C32, c: *mut C32,
                        ldc: usize, c_len: usize, prec: i32, err: *mut RbError) -> i32;
        pub fn rb_zgemm(transa: i32, transb: i32, m: usize, n: usize, k: usize, alpha: C64, a: *const C64,
                        lda: usize, a_len: usize, b: *const C64, ldb: usize, b_len: usize, beta: C64, c: *mut C64,
                        ldc: usize, c_len: usize, prec: i32, err: *mut RbError) -> i32;
        // level3::syrk / symm / trsm (src/level3.rs:236-520)
        pub fn rb_ssyrk(uplo: i32, trans: i32, n: usize, k: usize, alpha: f32, a: *const f32, lda: usize,
                        a_len: usize, beta: f32, c: *mut f32, ldc: usize, c_len: usize, err: *mut RbError) -> i32;
        pub fn rb_dsyrk(uplo: i32, trans: i32, n: usize, k: usize, alpha: f64, a: *const f64, lda: usize,
                        a_len: usize, beta: f64, c: *mut f64, ldc: usize, c_len: usize, err: *mut RbError) -> i32;
        pub fn rb_ssymm(side: i32, uplo: i32, m: usize, n: usize, alpha: f32, a: *const f32, lda: usize,
                        a_len: usize, b: *const f32, ldb: usize, b_len: usize, beta: f32, c: *mut f32, ldc: usize,
                        c_len: usize, err: *mut RbError) -> i32;
        pub fn rb_dsymm(side: i32, uplo: i32, m: usize, n: usize, alpha: f64, a: *const f64, lda: usize,
                        a_len: usize, b: *const f64, ldb: usize, b_len: usize, beta: f64, c: *mut f64, ldc: usize,
                        c_len: usize, err: *mut RbError) -> i32;
        pub fn rb_strsm(side: i32, uplo: i32, trans: i32, diag: i32, m: usize, n: usize, alpha: f32,
                        a: *const f32, lda: usize, a_len: usize, b: *mut f32, ldb: usize, b_len: usize,
                        err: *mut RbError) -> i32;
        pub fn rb_dtrsm(side: i32, uplo: i32, trans: i32, diag: i32, m: usize, n: usize, alpha: f64,
                        a: *const f64, lda: usize, a_len: usize, b: *mut f64, ldb: usize, b_len: usize,
                        err: *mut RbError) -> i32;
        // complex3::symm / hemm / trsm (src/complex3.rs:130-340)
        pub fn rb_csymm(side: i32, uplo: i32, m: usize, n: usize, alpha: C32, a: *const C32, lda: usize,
                        a_len: usize, b: *const C32, ldb: usize, b_len: usize, beta: C32, c: *mut C32, ldc: usize,
                        c_len: usize, err: *mut RbError) -> i32;
        pub fn rb_zsymm(side: i32, uplo: i32, m: usize, n: usize, alpha: C64, a: *const C64, lda: usize,
                        a_len: usize, b: *const C64, ldb: usize, b_len: usize, beta: C64, c: *mut C64, ldc: usize,
                        c_len: usize, err: *mut RbError) -> i32;
        pub fn rb_chemm(side: i32, uplo: i32, m: usize, n: usize, alpha: C32, a: *const C32, lda: usize,
                        a_len: usize, b: *const C32, ldb: usize, b_len: usize, beta: C32, c: *mut C32, ldc: usize,
                        c_len: usize, err: *mut RbError) -> i32;
        pub fn rb_zhemm(side: i32, uplo: i32, m: usize, n: usize, alpha: C64, a: *const C64, lda: usize,
                        a_len: usize, b: *const C64, ldb: usize, b_len: usize, beta: C64, c: *mut C64, ldc: usize,
                        c_len: usize, err: *mut RbError) -> i32;
        pub fn rb_ctrsm(side: i32, uplo: i32, trans: i32, diag: i32, m: usize, n: usize, alpha: C32,
                        a: *const C32, lda: usize, a_len: usize, b: *mut C32, ldb: usize, b_len: usize,
                        err: *mut RbError) -> i32;
        pub fn rb_ztrsm(side: i32, uplo: i32, trans: i32, diag: i32, m: usize, n: usize, alpha: C64,
                        a: *const C64, lda: usize, a_len: usize, b: *mut C64, ldb: usize, b_len: usize,
                        err: *mut RbError) -> i32;
        // level3::num_threads (src/level3.rs:11-17)
        pub fn rb_num_threads() -> usize;
        // device pointers, enqueued on a cudaStream_t (no rblas counterpart)
        pub fn rb_dgemm_dev(layout: i32, transa: i32, transb: i32, m: usize, n: usize, k: usize, alpha: f64,
                            a: *const f64, lda: usize, b: *const f64, ldb: usize, beta: f64, c: *mut f64,
                            ldc: usize, prec: i32, stream: *mut c_void, err: *mut RbError) -> i32;
        pub fn rb_sgemm_dev(layout: i32, transa: i32, transb: i32, m: usize, n: usize, k: usize, alpha: f32,
                            a: *const f32, lda: usize, b: *const f32, ldb: usize, beta: f32, c: *mut f32,
                            ldc: usize, prec: i32, stream: *mut c_void, err: *mut RbError) -> i32;
        pub fn rb_device_error(clear: i32, detail: *mut u32) -> i32;
    }

    // Level 1 and Level 2, host slices + lengths (src/level1.rs:17-163,
    // src/complex1.rs:8-112, src/level2.rs:11-89, src/complex2.rs:11-145)
    macro_rules! real_vec_ffi {
        ($t:ty, $axpy:ident, $scal:ident, $copy:ident, $swap:ident, $dot:ident, $asum:ident, $nrm2:ident,
         $gemv:ident, $ger:ident) => {
            extern "C" {
                pub fn $axpy(n: usize, alpha: $t, x: *const $t, incx: usize, x_len: usize, y: *mut $t, incy: usize,
                             y_len: usize, err: *mut RbError) -> i32;
                pub fn $scal(n: usize, alpha: $t, x: *mut $t, incx: usize, x_len: usize, err: *mut RbError) -> i32;
                pub fn $copy(n: usize, x: *const $t, incx: usize, x_len: usize, y: *mut $t, incy: usize,
                             y_len: usize, err: *mut RbError) -> i32;
                pub fn $swap(n: usize, x: *mut $t, incx: usize, x_len: usize, y: *mut $t, incy: usize, y_len: usize,
                             err: *mut RbError) -> i32;
                pub fn $dot(n: usize, x: *const $t, incx: usize, x_len: usize, y: *const $t, incy: usize,
                            y_len: usize, result: *mut $t, err: *mut RbError) -> i32;
                pub fn $asum(n: usize, x: *const $t, incx: usize, x_len: usize, result: *mut $t,
                             err: *mut RbError) -> i32;
                pub fn $nrm2(n: usize, x: *const $t, incx: usize, x_len: usize, result: *mut $t,
                             err: *mut RbError) -> i32;
                pub fn $gemv(layout: i32, trans: i32, m: usize, n: usize, alpha: $t, a: *const $t, lda: usize,
                             a_len: usize, x: *const $t, incx: usize, x_len: usize, beta: $t, y: *mut $t,
                             incy: usize, y_len: usize, err: *mut RbError) -> i32;
                pub fn $ger(layout: i32, m: usize, n: usize, alpha: $t, x: *const $t, incx: usize, x_len: usize,
                            y: *const $t, incy: usize, y_len: usize, a: *mut $t, lda: usize, a_len: usize,
                            err: *mut RbError) -> i32;
            }
        };
    }
    real_vec_ffi!(f32, rb_saxpy, rb_sscal, rb_scopy, rb_sswap, rb_sdot, rb_sasum, rb_snrm2, rb_sgemv, rb_sger);
    real_vec_ffi!(f64, rb_daxpy, rb_dscal, rb_dcopy, rb_dswap, rb_ddot, rb_dasum, rb_dnrm2, rb_dgemv, rb_dger);

    macro_rules! complex_vec_ffi {
        ($t:ty, $r:ty, $axpy:ident, $scal:ident, $dotu:ident, $dotc:ident, $nrm2:ident, $gemv:ident,
         $geru:ident, $gerc:ident) => {
            extern "C" {
                pub fn $axpy(n: usize, alpha: $t, x: *const $t, incx: usize, x_len: usize, y: *mut $t, incy: usize,
                             y_len: usize, err: *mut RbError) -> i32;
                pub fn $scal(n: usize, alpha: $t, x: *mut $t, incx: usize, x_len: usize, err: *mut RbError) -> i32;
                pub fn $dotu(n: usize, x: *const $t, incx: usize, x_len: usize, y: *const $t, incy: usize,
                             y_len: usize, result: *mut $t, err: *mut RbError) -> i32;
                pub fn $dotc(n: usize, x: *const $t, incx: usize, x_len: usize, y: *const $t, incy: usize,
                             y_len: usize, result: *mut $t, err: *mut RbError) -> i32;
                pub fn $nrm2(n: usize, x: *const $t, incx: usize, x_len: usize, result: *mut $r,
                             err: *mut RbError) -> i32;
                pub fn $gemv(layout: i32, trans: i32, m: usize, n: usize, alpha: $t, a: *const $t, lda: usize,
                             a_len: usize, x: *const $t, incx: usize, x_len: usize, beta: $t, y: *mut $t,
                             incy: usize, y_len: usize, err: *mut RbError) -> i32;
                pub fn $geru(layout: i32, m: usize, n: usize, alpha: $t, x: *const $t, incx: usize, x_len: usize,
                             y: *const $t, incy: usize, y_len: usize, a: *mut $t, lda: usize, a_len: usize,
                             err: *mut RbError) -> i32;
                pub fn $gerc(layout: i32, m: usize, n: usize, alpha: $t, x: *const $t, incx: usize, x_len: usize,
                             y: *const $t, incy: usize, y_len: usize, a: *mut $t, lda: usize, a_len: usize,
                             err: *mut RbError) -> i32;
            }
        };
    }
    complex_vec_ffi!(C32, f32, rb_caxpy, rb_cscal, rb_cdotu, rb_cdotc, rb_scnrm2, rb_cgemv, rb_cgeru, rb_cgerc);
    complex_vec_ffi!(C64, f64, rb_zaxpy, rb_zscal, rb_zdotu, rb_zdotc, rb_dznrm2, rb_zgemv, rb_zgeru, rb_zgerc);
}

use ffi::RbError;

fn layout(l: Layout) -> i32 {
    match l {
        Layout::RowMajor => 0,
        Layout::ColMajor => 1,
    }
}
fn trans(t: Transpose) -> i32 {
    match t {
        Transpose::None => 0,
        Transpose::Trans => 1,
        Transpose::ConjTrans => 2,
    }
}
fn uplo(u: Uplo) -> i32 {
    match u {
        Uplo::Upper => 0,
        Uplo::Lower => 1,
    }
}
fn side(s: Side) -> i32 {
    match s {
        Side::Left => 0,
        Side::Right => 1,
    }
}
fn diag(d: Diag) -> i32 {
    match d {
        Diag::NonUnit => 0,
        Diag::Unit => 1,
    }
}

/// `rb_error` -> the matching rblas error (`src/error.rs:15-39`) or a device error.
fn check(status: i32, e: &RbError) -> Result<(), Error> {
    let which: &'static str = match e.which {
        b'a' => "a",
        b'b' => "b",
        b'c' => "c",
        b'x' => "x",
        b'y' => "y",
        _ => "?",
    };
    match status {
        0 => Ok(()),
        1 => Err(Error::Blas(BlasError::InvalidLeadingDim { which, got: e.got as usize, min: e.min_or_need as usize })),
        2 => Err(Error::Blas(BlasError::BufferTooSmall { which, got: e.got as usize, need: e.min_or_need as usize })),
        3 => Err(Error::Blas(BlasError::ZeroStride { which })),
        code => Err(Error::Device { code, cuda_error: e.cuda_error, detail: e.got }),
    }
}

/// The rblas-shaped result: argument errors returned, device failures raised.
fn blas(r: Result<(), Error>) -> rblas::Result<()> {
    match r {
        Ok(()) => Ok(()),
        Err(Error::Blas(e)) => Err(e),
        Err(e) => panic!("{e}"),
    }
}

/// Element types of the real routines (`rblas::Float` restricted to f32 / f64).
pub trait GpuFloat: Copy {
    #[doc(hidden)]
    #[allow(clippy::too_many_arguments)]
    unsafe fn gemm_raw(l: i32, ta: i32, tb: i32, m: usize, n: usize, k: usize, alpha: Self, a: &[Self], lda: usize,
                       b: &[Self], ldb: usize, beta: Self, c: &mut [Self], ldc: usize, prec: i32,
                       e: &mut RbError) -> i32;
    #[doc(hidden)]
    #[allow(clippy::too_many_arguments)]
    unsafe fn syrk_raw(u: i32, t: i32, n: usize, k: usize, alpha: Self, a: &[Self], lda: usize, beta: Self,
                       c: &mut [Self], ldc: usize, e: &mut RbError) -> i32;
    #[doc(hidden)]
    #[allow(clippy::too_many_arguments)]
    unsafe fn symm_raw(s: i32, u: i32, m: usize, n: usize, alpha: Self, a: &[Self], lda: usize, b: &[Self],
                       ldb: usize, beta: Self, c: &mut [Self], ldc: usize, e: &mut RbError) -> i32;
    #[doc(hidden)]
    #[allow(clippy::too_many_arguments)]
    unsafe fn trsm_raw(s: i32, u: i32, t: i32, d: i32, m: usize, n: usize, alpha: Self, a: &[Self], lda: usize,
                       b: &mut [Self], ldb: usize, e: &mut RbError) -> i32;
}

macro_rules! real_impl {
    ($t:ty, $gemm:ident, $syrk:ident, $symm:ident, $trsm:ident) => {
        impl GpuFloat for $t {
            unsafe fn gemm_raw(l: i32, ta: i32, tb: i32, m: usize, n: usize, k: usize, alpha: Self, a: &[Self],
                               lda: usize, b: &[Self], ldb: usize, beta: Self, c: &mut [Self], ldc: usize, prec: i32,
                               e: &mut RbError) -> i32 {
                ffi::$gemm(l, ta, tb, m, n, k, alpha, a.as_ptr(), lda, a.len(), b.as_ptr(), ldb, b.len(), beta,
                           c.as_mut_ptr(), ldc, c.len(), prec, e)
            }
            unsafe fn syrk_raw(u: i32, t: i32, n: usize, k: usize, alpha: Self, a: &[Self], lda: usize, beta: Self,
                               c: &mut [Self], ldc: usize, e: &mut RbError) -> i32 {
                ffi::$syrk(u, t, n, k, alpha, a.as_ptr(), lda, a.len(), beta, c.as_mut_ptr(), ldc, c.len(), e)
            }
            unsafe fn symm_raw(s: i32, u: i32, m: usize, n: usize, alpha: Self, a: &[Self], lda: usize, b: &[Self],
                               ldb: usize, beta: Self, c: &mut [Self], ldc: usize, e: &mut RbError) -> i32 {
                ffi::$symm(s, u, m, n, alpha, a.as_ptr(), lda, a.len(), b.as_ptr(), ldb, b.len(), beta,
                           c.as_mut_ptr(), ldc, c.len(), e)
            }
            unsafe fn trsm_raw(s: i32, u: i32, t: i32, d: i32, m: usize, n: usize, alpha: Self, a: &[Self],
                               lda: usize, b: &mut [Self], ldb: usize, e: &mut RbError) -> i32 {
                ffi::$trsm(s, u, t, d, m, n, alpha, a.as_ptr(), lda, a.len(), b.as_mut_ptr(), ldb, b.len(), e)
            }
        }
    };
}
real_impl!(f32, rb_sgemm_prec, rb_ssyrk, rb_ssymm, rb_strsm);
real_impl!(f64, rb_dgemm_prec, rb_dsyrk, rb_dsymm, rb_dtrsm);

/// `rblas::level3` on the GPU.
pub mod level3 {
    use super::*;

    /// level3::num_threads (`src/level3.rs:11-17`): the device's SM count
    /// (every persistent GEMM kernel runs one CTA per SM); 1 without a device.
    pub fn num_threads() -> usize {
        unsafe { ffi::rb_num_threads() }
    }

    /// level3::try_gemm with an arithmetic form; device failures as [`Error::Device`].
    #[allow(clippy::too_many_arguments)]
    pub fn try_gemm_prec<T: GpuFloat>(l: Layout, ta: Transpose, tb: Transpose, m: usize, n: usize, k: usize,
                                      alpha: T, a: &[T], lda: usize, b: &[T], ldb: usize, beta: T, c: &mut [T],
                                      ldc: usize, prec: Precision) -> Result<(), Error> {
        let mut e = RbError::default();
        let st = unsafe {
            T::gemm_raw(layout(l), trans(ta), trans(tb), m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, prec as i32,
                        &mut e)
        };
        check(st, &e)
    }

    /// Drop-in for `rblas::level3::try_gemm` (`src/level3.rs:68-103`).
    #[allow(clippy::too_many_arguments)]
    pub fn try_gemm<T: GpuFloat>(l: Layout, ta: Transpose, tb: Transpose, m: usize, n: usize, k: usize, alpha: T,
                                 a: &[T], lda: usize, b: &[T], ldb: usize, beta: T, c: &mut [T],
                                 ldc: usize) -> rblas::Result<()> {
        blas(try_gemm_prec(l, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, Precision::Plain))
    }

    /// Drop-in for `rblas::level3::gemm` (`src/level3.rs:32-62`): panics where rblas panics.
    #[allow(clippy::too_many_arguments)]
    pub fn gemm<T: GpuFloat>(l: Layout, ta: Transpose, tb: Transpose, m: usize, n: usize, k: usize, alpha: T,
                             a: &[T], lda: usize, b: &[T], ldb: usize, beta: T, c: &mut [T], ldc: usize) {
        try_gemm(l, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc).unwrap()
    }

    /// Drop-in for `rblas::level3::syrk` (`src/level3.rs:236-294`).
    #[allow(clippy::too_many_arguments)]
    pub fn syrk<T: GpuFloat>(u: Uplo, t: Transpose, n: usize, k: usize, alpha: T, a: &[T], lda: usize, beta: T,
                             c: &mut [T], ldc: usize) {
        let mut e = RbError::default();
        let st = unsafe { T::syrk_raw(uplo(u), trans(t), n, k, alpha, a, lda, beta, c, ldc, &mut e) };
        blas(check(st, &e)).unwrap()
    }

    /// Drop-in for `rblas::level3::symm` (`src/level3.rs:301-354`).
    #[allow(clippy::too_many_arguments)]
    pub fn symm<T: GpuFloat>(s: Side, u: Uplo, m: usize, n: usize, alpha: T, a: &[T], lda: usize, b: &[T],
                             ldb: usize, beta: T, c: &mut [T], ldc: usize) {
        let mut e = RbError::default();
        let st = unsafe { T::symm_raw(side(s), uplo(u), m, n, alpha, a, lda, b, ldb, beta, c, ldc, &mut e) };
        blas(check(st, &e)).unwrap()
    }

    /// Drop-in for `rblas::level3::trsm` (`src/level3.rs:390-520`).
    #[allow(clippy::too_many_arguments)]
    pub fn trsm<T: GpuFloat>(s: Side, u: Uplo, t: Transpose, d: Diag, m: usize, n: usize, alpha: T, a: &[T],
                             lda: usize, b: &mut [T], ldb: usize) {
        let mut e = RbError::default();
        let st = unsafe { T::trsm_raw(side(s), uplo(u), trans(t), diag(d), m, n, alpha, a, lda, b, ldb, &mut e) };
        blas(check(st, &e)).unwrap()
    }

    /// Device-pointer f64 GEMM enqueued on a `cudaStream_t` (no rblas
    /// counterpart). Returns once the work is enqueued; read device-side
    /// failures afterwards with [`device_error`].
    ///
    /// # Safety
    /// `a`, `b`, `c` must be device pointers to matrices of the stated shapes
    /// and leading dimensions, valid until the stream reaches the work.
    #[allow(clippy::too_many_arguments)]
    pub unsafe fn dgemm_dev(l: Layout, ta: Transpose, tb: Transpose, m: usize, n: usize, k: usize, alpha: f64,
                            a: *const f64, lda: usize, b: *const f64, ldb: usize, beta: f64, c: *mut f64,
                            ldc: usize, prec: Precision, stream: *mut c_void) -> Result<(), Error> {
        let mut e = RbError::default();
        let st = ffi::rb_dgemm_dev(layout(l), trans(ta), trans(tb), m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                                   prec as i32, stream, &mut e);
        check(st, &e)
    }

    /// The current device's error word (after `*_dev` calls): Ok when clear.
    pub fn device_error(clear: bool) -> Result<(), Error> {
        let mut w = 0u32;
        let st = unsafe { ffi::rb_device_error(clear as i32, &mut w) };
        if st == 0 {
            Ok(())
        } else {
            Err(Error::Device { code: st, cuda_error: 0, detail: w as u64 })
        }
    }
}

/// Element types of the complex routines (`Complex<f32>` / `Complex<f64>`).
pub trait GpuComplex: Copy {
    #[doc(hidden)]
    #[allow(clippy::too_many_arguments)]
    unsafe fn gemm_raw(ta: i32, tb: i32, m: usize, n: usize, k: usize, alpha: Self, a: &[Self], lda: usize,
                       b: &[Self], ldb: usize, beta: Self, c: &mut [Self], ldc: usize, prec: i32,
                       e: &mut RbError) -> i32;
    #[doc(hidden)]
    #[allow(clippy::too_many_arguments)]
    unsafe fn hesy_raw(herm: bool, s: i32, u: i32, m: usize, n: usize, alpha: Self, a: &[Self], lda: usize,
                       b: &[Self], ldb: usize, beta: Self, c: &mut [Self], ldc: usize, e: &mut RbError) -> i32;
    #[doc(hidden)]
    #[allow(clippy::too_many_arguments)]
    unsafe fn trsm_raw(s: i32, u: i32, t: i32, d: i32, m: usize, n: usize, alpha: Self, a: &[Self], lda: usize,
                       b: &mut [Self], ldb: usize, e: &mut RbError) -> i32;
}

macro_rules! complex_impl {
    ($t:ty, $gemm:ident, $symm:ident, $hemm:ident, $trsm:ident) => {
        impl GpuComplex for $t {
            unsafe fn gemm_raw(ta: i32, tb: i32, m: usize, n: usize, k: usize, alpha: Self, a: &[Self], lda: usize,
                               b: &[Self], ldb: usize, beta: Self, c: &mut [Self], ldc: usize, prec: i32,
                               e: &mut RbError) -> i32 {
                ffi::$gemm(ta, tb, m, n, k, alpha, a.as_ptr(), lda, a.len(), b.as_ptr(), ldb, b.len(), beta,
                           c.as_mut_ptr(), ldc, c.len(), prec, e)
            }
            unsafe fn hesy_raw(herm: bool, s: i32, u: i32, m: usize, n: usize, alpha: Self, a: &[Self], lda: usize,
                               b: &[Self], ldb: usize, beta: Self, c: &mut [Self], ldc: usize,
                               e: &mut RbError) -> i32 {
                let f = if herm { ffi::$hemm } else { ffi::$symm };
                f(s, u, m, n, alpha, a.as_ptr(), lda, a.len(), b.as_ptr(), ldb, b.len(), beta, c.as_mut_ptr(), ldc,
                  c.len(), e)
            }
            unsafe fn trsm_raw(s: i32, u: i32, t: i32, d: i32, m: usize, n: usize, alpha: Self, a: &[Self],
                               lda: usize, b: &mut [Self], ldb: usize, e: &mut RbError) -> i32 {
                ffi::$trsm(s, u, t, d, m, n, alpha, a.as_ptr(), lda, a.len(), b.as_mut_ptr(), ldb, b.len(), e)
            }
        }
    };
}
complex_impl!(C32, rb_cgemm, rb_csymm, rb_chemm, rb_ctrsm);
complex_impl!(C64, rb_zgemm, rb_zsymm, rb_zhemm, rb_ztrsm);

/// `rblas::complex3` on the GPU (column-major, like rblas's).
pub mod complex3 {
    use super::*;

    /// complex3::gemm with an arithmetic form (BF16X3 / BF16X6 for C32, Ozaki for C64).
    #[allow(clippy::too_many_arguments)]
    pub fn try_gemm_prec<T: GpuComplex>(ta: Transpose, tb: Transpose, m: usize, n: usize, k: usize, alpha: T,
                                        a: &[T], lda: usize, b: &[T], ldb: usize, beta: T, c: &mut [T], ldc: usize,
                                        prec: Precision) -> Result<(), Error> {
        let mut e = RbError::default();
        let st = unsafe {
            T::gemm_raw(trans(ta), trans(tb), m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, prec as i32, &mut e)
        };
        check(st, &e)
    }

    /// Drop-in for `rblas::complex3::gemm` (`src/complex3.rs:27-74`).
    #[allow(clippy::too_many_arguments)]
    pub fn gemm<T: GpuComplex>(ta: Transpose, tb: Transpose, m: usize, n: usize, k: usize, alpha: T, a: &[T],
                               lda: usize, b: &[T], ldb: usize, beta: T, c: &mut [T], ldc: usize) {
        blas(try_gemm_prec(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, Precision::Plain)).unwrap()
    }

    /// Drop-in for `rblas::complex3::symm` (`src/complex3.rs:130-145`).
    #[allow(clippy::too_many_arguments)]
    pub fn symm<T: GpuComplex>(s: Side, u: Uplo, m: usize, n: usize, alpha: T, a: &[T], lda: usize, b: &[T],
                               ldb: usize, beta: T, c: &mut [T], ldc: usize) {
        let mut e = RbError::default();
        let st = unsafe { T::hesy_raw(false, side(s), uplo(u), m, n, alpha, a, lda, b, ldb, beta, c, ldc, &mut e) };
        blas(check(st, &e)).unwrap()
    }

    /// Drop-in for `rblas::complex3::hemm` (`src/complex3.rs:151-166`).
    #[allow(clippy::too_many_arguments)]
    pub fn hemm<T: GpuComplex>(s: Side, u: Uplo, m: usize, n: usize, alpha: T, a: &[T], lda: usize, b: &[T],
                               ldb: usize, beta: T, c: &mut [T], ldc: usize) {
        let mut e = RbError::default();
        let st = unsafe { T::hesy_raw(true, side(s), uplo(u), m, n, alpha, a, lda, b, ldb, beta, c, ldc, &mut e) };
        blas(check(st, &e)).unwrap()
    }

    /// Drop-in for `rblas::complex3::trsm` (`src/complex3.rs:252-340`).
    #[allow(clippy::too_many_arguments)]
    pub fn trsm<T: GpuComplex>(s: Side, u: Uplo, t: Transpose, d: Diag, m: usize, n: usize, alpha: T, a: &[T],
                               lda: usize, b: &mut [T], ldb: usize) {
        let mut e = RbError::default();
        let st = unsafe { T::trsm_raw(side(s), uplo(u), trans(t), diag(d), m, n, alpha, a, lda, b, ldb, &mut e) };
        blas(check(st, &e)).unwrap()
    }
}

/// rblas's Level-1 and Level-2 routines panic on arguments they cannot use
/// (a stride of zero, a slice shorter than the strided range); so do these,
/// with the library's message. Device failures panic too.
fn must(status: i32, e: &RbError) {
    if let Err(err) = check(status, e) {
        panic!("{err}");
    }
}

/// Element types of the real Level-1 / Level-2 routines (f32 / f64).
pub trait GpuVecFloat: GpuFloat + Default {
    #[doc(hidden)]
    unsafe fn axpy_raw(n: usize, alpha: Self, x: &[Self], incx: usize, y: &mut [Self], incy: usize,
                       e: &mut RbError) -> i32;
    #[doc(hidden)]
    unsafe fn scal_raw(n: usize, alpha: Self, x: &mut [Self], incx: usize, e: &mut RbError) -> i32;
    #[doc(hidden)]
    unsafe fn copy_raw(n: usize, x: &[Self], incx: usize, y: &mut [Self], incy: usize, e: &mut RbError) -> i32;
    #[doc(hidden)]
    unsafe fn swap_raw(n: usize, x: &mut [Self], incx: usize, y: &mut [Self], incy: usize, e: &mut RbError) -> i32;
    #[doc(hidden)]
    unsafe fn dot_raw(n: usize, x: &[Self], incx: usize, y: &[Self], incy: usize, r: &mut Self,
                      e: &mut RbError) -> i32;
    #[doc(hidden)]
    unsafe fn asum_raw(n: usize, x: &[Self], incx: usize, r: &mut Self, e: &mut RbError) -> i32;
    #[doc(hidden)]
    unsafe fn nrm2_raw(n: usize, x: &[Self], incx: usize, r: &mut Self, e: &mut RbError) -> i32;
    #[doc(hidden)]
    #[allow(clippy::too_many_arguments)]
    unsafe fn gemv_raw(l: i32, t: i32, m: usize, n: usize, alpha: Self, a: &[Self], lda: usize, x: &[Self],
                       incx: usize, beta: Self, y: &mut [Self], incy: usize, e: &mut RbError) -> i32;
    #[doc(hidden)]
    #[allow(clippy::too_many_arguments)]
    unsafe fn ger_raw(l: i32, m: usize, n: usize, alpha: Self, x: &[Self], incx: usize, y: &[Self], incy: usize,
                      a: &mut [Self], lda: usize, e: &mut RbError) -> i32;
}

macro_rules! real_vec_impl {
    ($t:ty, $axpy:ident, $scal:ident, $copy:ident, $swap:ident, $dot:ident, $asum:ident, $nrm2:ident,
     $gemv:ident, $ger:ident) => {
        impl GpuVecFloat for $t {
            unsafe fn axpy_raw(n: usize, alpha: Self, x: &[Self], incx: usize, y: &mut [Self], incy: usize,
                               e: &mut RbError) -> i32 {
                ffi::$axpy(n, alpha, x.as_ptr(), incx, x.len(), y.as_mut_ptr(), incy, y.len(), e)
            }
            unsafe fn scal_raw(n: usize, alpha: Self, x: &mut [Self], incx: usize, e: &mut RbError) -> i32 {
                ffi::$scal(n, alpha, x.as_mut_ptr(), incx, x.len(), e)
            }
            unsafe fn copy_raw(n: usize, x: &[Self], incx: usize, y: &mut [Self], incy: usize,
                               e: &mut RbError) -> i32 {
                ffi::$copy(n, x.as_ptr(), incx, x.len(), y.as_mut_ptr(), incy, y.len(), e)
            }
            unsafe fn swap_raw(n: usize, x: &mut [Self], incx: usize, y: &mut [Self], incy: usize,
                               e: &mut RbError) -> i32 {
                ffi::$swap(n, x.as_mut_ptr(), incx, x.len(), y.as_mut_ptr(), incy, y.len(), e)
            }
            unsafe fn dot_raw(n: usize, x: &[Self], incx: usize, y: &[Self], incy: usize, r: &mut Self,
                              e: &mut RbError) -> i32 {
                ffi::$dot(n, x.as_ptr(), incx, x.len(), y.as_ptr(), incy, y.len(), r, e)
            }
            unsafe fn asum_raw(n: usize, x: &[Self], incx: usize, r: &mut Self, e: &mut RbError) -> i32 {
                ffi::$asum(n, x.as_ptr(), incx, x.len(), r, e)
            }
            unsafe fn nrm2_raw(n: usize, x: &[Self], incx: usize, r: &mut Self, e: &mut RbError) -> i32 {
                ffi::$nrm2(n, x.as_ptr(), incx, x.len(), r, e)
            }
            unsafe fn gemv_raw(l: i32, t: i32, m: usize, n: usize, alpha: Self, a: &[Self], lda: usize, x: &[Self],
                               incx: usize, beta: Self, y: &mut [Self], incy: usize, e: &mut RbError) -> i32 {
                ffi::$gemv(l, t, m, n, alpha, a.as_ptr(), lda, a.len(), x.as_ptr(), incx, x.len(), beta,
                           y.as_mut_ptr(), incy, y.len(), e)
            }
            unsafe fn ger_raw(l: i32, m: usize, n: usize, alpha: Self, x: &[Self], incx: usize, y: &[Self],
                              incy: usize, a: &mut [Self], lda: usize, e: &mut RbError) -> i32 {
                ffi::$ger(l, m, n, alpha, x.as_ptr(), incx, x.len(), y.as_ptr(), incy, y.len(), a.as_mut_ptr(), lda,
                          a.len(), e)
            }
        }
    };
}
real_vec_impl!(f32, rb_saxpy, rb_sscal, rb_scopy, rb_sswap, rb_sdot, rb_sasum, rb_snrm2, rb_sgemv, rb_sger);
real_vec_impl!(f64, rb_daxpy, rb_dscal, rb_dcopy, rb_dswap, rb_ddot, rb_dasum, rb_dnrm2, rb_dgemv, rb_dger);

/// `rblas::level1` on the GPU (strided vectors; each call copies them to the
/// device and back).
pub mod level1 {
    use super::*;

    /// Drop-in for `rblas::level1::axpy` (`src/level1.rs:17-41`): y := alpha*x + y.
    pub fn axpy<T: GpuVecFloat>(n: usize, alpha: T, x: &[T], incx: usize, y: &mut [T], incy: usize) {
        let mut e = RbError::default();
        must(unsafe { T::axpy_raw(n, alpha, x, incx, y, incy, &mut e) }, &e)
    }

    /// Drop-in for `rblas::level1::dot` (`src/level1.rs:45-66`).
    pub fn dot<T: GpuVecFloat>(n: usize, x: &[T], incx: usize, y: &[T], incy: usize) -> T {
        let (mut e, mut r) = (RbError::default(), T::default());
        must(unsafe { T::dot_raw(n, x, incx, y, incy, &mut r, &mut e) }, &e);
        r
    }

    /// Drop-in for `rblas::level1::scal` (`src/level1.rs:70-86`): x := alpha*x.
    pub fn scal<T: GpuVecFloat>(n: usize, alpha: T, x: &mut [T], incx: usize) {
        let mut e = RbError::default();
        must(unsafe { T::scal_raw(n, alpha, x, incx, &mut e) }, &e)
    }

    /// Drop-in for `rblas::level1::nrm2` (`src/level1.rs:96-123`).
    pub fn nrm2<T: GpuVecFloat>(n: usize, x: &[T], incx: usize) -> T {
        let (mut e, mut r) = (RbError::default(), T::default());
        must(unsafe { T::nrm2_raw(n, x, incx, &mut r, &mut e) }, &e);
        r
    }

    /// Drop-in for `rblas::level1::asum` (`src/level1.rs:127-135`).
    pub fn asum<T: GpuVecFloat>(n: usize, x: &[T], incx: usize) -> T {
        let (mut e, mut r) = (RbError::default(), T::default());
        must(unsafe { T::asum_raw(n, x, incx, &mut r, &mut e) }, &e);
        r
    }

    /// Drop-in for `rblas::level1::copy` (`src/level1.rs:139-151`): y := x.
    pub fn copy<T: GpuVecFloat>(n: usize, x: &[T], incx: usize, y: &mut [T], incy: usize) {
        let mut e = RbError::default();
        must(unsafe { T::copy_raw(n, x, incx, y, incy, &mut e) }, &e)
    }

    /// Drop-in for `rblas::level1::swap` (`src/level1.rs:155-163`).
    pub fn swap<T: GpuVecFloat>(n: usize, x: &mut [T], incx: usize, y: &mut [T], incy: usize) {
        let mut e = RbError::default();
        must(unsafe { T::swap_raw(n, x, incx, y, incy, &mut e) }, &e)
    }
}

/// `rblas::level2` on the GPU.
pub mod level2 {
    use super::*;

    /// Drop-in for `rblas::level2::gemv` (`src/level2.rs:11-61`): y := alpha*op(A)*x + beta*y.
    #[allow(clippy::too_many_arguments)]
    pub fn gemv<T: GpuVecFloat>(l: Layout, t: Transpose, m: usize, n: usize, alpha: T, a: &[T], lda: usize,
                                x: &[T], incx: usize, beta: T, y: &mut [T], incy: usize) {
        let mut e = RbError::default();
        must(unsafe { T::gemv_raw(layout(l), trans(t), m, n, alpha, a, lda, x, incx, beta, y, incy, &mut e) }, &e)
    }

    /// Drop-in for `rblas::level2::ger` (`src/level2.rs:65-88`): A := alpha*x*y^T + A.
    #[allow(clippy::too_many_arguments)]
    pub fn ger<T: GpuVecFloat>(l: Layout, m: usize, n: usize, alpha: T, x: &[T], incx: usize, y: &[T], incy: usize,
                               a: &mut [T], lda: usize) {
        let mut e = RbError::default();
        must(unsafe { T::ger_raw(layout(l), m, n, alpha, x, incx, y, incy, a, lda, &mut e) }, &e)
    }
}

/// Element types of the complex Level-1 / Level-2 routines (C32 / C64).
pub trait GpuVecComplex: GpuComplex {
    /// The real type of `nrm2`'s result.
    type Real: Copy + Default;
    #[doc(hidden)]
    fn zero() -> Self;
    #[doc(hidden)]
    unsafe fn axpy_raw(n: usize, alpha: Self, x: &[Self], incx: usize, y: &mut [Self], incy: usize,
                       e: &mut RbError) -> i32;
    #[doc(hidden)]
    unsafe fn scal_raw(n: usize, alpha: Self, x: &mut [Self], incx: usize, e: &mut RbError) -> i32;
    #[doc(hidden)]
    #[allow(clippy::too_many_arguments)]
    unsafe fn dot_raw(conj: bool, n: usize, x: &[Self], incx: usize, y: &[Self], incy: usize, r: &mut Self,
                      e: &mut RbError) -> i32;
    #[doc(hidden)]
    unsafe fn nrm2_raw(n: usize, x: &[Self], incx: usize, r: &mut Self::Real, e: &mut RbError) -> i32;
    #[doc(hidden)]
    #[allow(clippy::too_many_arguments)]
    unsafe fn gemv_raw(l: i32, t: i32, m: usize, n: usize, alpha: Self, a: &[Self], lda: usize, x: &[Self],
                       incx: usize, beta: Self, y: &mut [Self], incy: usize, e: &mut RbError) -> i32;
    #[doc(hidden)]
    #[allow(clippy::too_many_arguments)]
    unsafe fn ger_raw(conj: bool, l: i32, m: usize, n: usize, alpha: Self, x: &[Self], incx: usize, y: &[Self],
                      incy: usize, a: &mut [Self], lda: usize, e: &mut RbError) -> i32;
}

macro_rules! complex_vec_impl {
    ($t:ty, $r:ty, $axpy:ident, $scal:ident, $dotu:ident, $dotc:ident, $nrm2:ident, $gemv:ident, $geru:ident,
     $gerc:ident) => {
        impl GpuVecComplex for $t {
            type Real = $r;
            fn zero() -> Self {
                Complex::new(0.0, 0.0)
            }
            unsafe fn axpy_raw(n: usize, alpha: Self, x: &[Self], incx: usize, y: &mut [Self], incy: usize,
                               e: &mut RbError) -> i32 {
                ffi::$axpy(n, alpha, x.as_ptr(), incx, x.len(), y.as_mut_ptr(), incy, y.len(), e)
            }
            unsafe fn scal_raw(n: usize, alpha: Self, x: &mut [Self], incx: usize, e: &mut RbError) -> i32 {
                ffi::$scal(n, alpha, x.as_mut_ptr(), incx, x.len(), e)
            }
            unsafe fn dot_raw(conj: bool, n: usize, x: &[Self], incx: usize, y: &[Self], incy: usize, r: &mut Self,
                              e: &mut RbError) -> i32 {
                let f = if conj { ffi::$dotc } else { ffi::$dotu };
                f(n, x.as_ptr(), incx, x.len(), y.as_ptr(), incy, y.len(), r, e)
            }
            unsafe fn nrm2_raw(n: usize, x: &[Self], incx: usize, r: &mut $r, e: &mut RbError) -> i32 {
                ffi::$nrm2(n, x.as_ptr(), incx, x.len(), r, e)
            }
            unsafe fn gemv_raw(l: i32, t: i32, m: usize, n: usize, alpha: Self, a: &[Self], lda: usize, x: &[Self],
                               incx: usize, beta: Self, y: &mut [Self], incy: usize, e: &mut RbError) -> i32 {
                ffi::$gemv(l, t, m, n, alpha, a.as_ptr(), lda, a.len(), x.as_ptr(), incx, x.len(), beta,
                           y.as_mut_ptr(), incy, y.len(), e)
            }
            unsafe fn ger_raw(conj: bool, l: i32, m: usize, n: usize, alpha: Self, x: &[Self], incx: usize,
                              y: &[Self], incy: usize, a: &mut [Self], lda: usize, e: &mut RbError) -> i32 {
                let f = if conj { ffi::$gerc } else { ffi::$geru };
                f(l, m, n, alpha, x.as_ptr(), incx, x.len(), y.as_ptr(), incy, y.len(), a.as_mut_ptr(), lda, a.len(),
                  e)
            }
        }
    };
}
complex_vec_impl!(C32, f32, rb_caxpy, rb_cscal, rb_cdotu, rb_cdotc, rb_scnrm2, rb_cgemv, rb_cgeru, rb_cgerc);
complex_vec_impl!(C64, f64, rb_zaxpy, rb_zscal, rb_zdotu, rb_zdotc, rb_dznrm2, rb_zgemv, rb_zgeru, rb_zgerc);

/// `rblas::complex1` on the GPU.
pub mod complex1 {
    use super::*;

    /// Drop-in for `rblas::complex1::axpy` (`src/complex1.rs:8-27`).
    pub fn axpy<T: GpuVecComplex>(n: usize, alpha: T, x: &[T], incx: usize, y: &mut [T], incy: usize) {
        let mut e = RbError::default();
        must(unsafe { T::axpy_raw(n, alpha, x, incx, y, incy, &mut e) }, &e)
    }

    /// Drop-in for `rblas::complex1::dotu` (`src/complex1.rs:31-47`): x^T y.
    pub fn dotu<T: GpuVecComplex>(n: usize, x: &[T], incx: usize, y: &[T], incy: usize) -> T {
        let (mut e, mut r) = (RbError::default(), T::zero());
        must(unsafe { T::dot_raw(false, n, x, incx, y, incy, &mut r, &mut e) }, &e);
        r
    }

    /// Drop-in for `rblas::complex1::dotc` (`src/complex1.rs:51-67`): x^H y.
    pub fn dotc<T: GpuVecComplex>(n: usize, x: &[T], incx: usize, y: &[T], incy: usize) -> T {
        let (mut e, mut r) = (RbError::default(), T::zero());
        must(unsafe { T::dot_raw(true, n, x, incx, y, incy, &mut r, &mut e) }, &e);
        r
    }

    /// Drop-in for `rblas::complex1::scal` (`src/complex1.rs:71-81`).
    pub fn scal<T: GpuVecComplex>(n: usize, alpha: T, x: &mut [T], incx: usize) {
        let mut e = RbError::default();
        must(unsafe { T::scal_raw(n, alpha, x, incx, &mut e) }, &e)
    }

    /// Drop-in for `rblas::complex1::nrm2` (`src/complex1.rs:86-112`).
    pub fn nrm2<T: GpuVecComplex>(n: usize, x: &[T], incx: usize) -> T::Real {
        let (mut e, mut r) = (RbError::default(), T::Real::default());
        must(unsafe { T::nrm2_raw(n, x, incx, &mut r, &mut e) }, &e);
        r
    }
}

/// `rblas::complex2` on the GPU.
pub mod complex2 {
    use super::*;

    /// Drop-in for `rblas::complex2::gemv` (`src/complex2.rs:11-76`); ConjTrans conjugates A.
    #[allow(clippy::too_many_arguments)]
    pub fn gemv<T: GpuVecComplex>(l: Layout, t: Transpose, m: usize, n: usize, alpha: T, a: &[T], lda: usize,
                                  x: &[T], incx: usize, beta: T, y: &mut [T], incy: usize) {
        let mut e = RbError::default();
        must(unsafe { T::gemv_raw(layout(l), trans(t), m, n, alpha, a, lda, x, incx, beta, y, incy, &mut e) }, &e)
    }

    /// Drop-in for `rblas::complex2::geru` (`src/complex2.rs:80-93`): A := alpha*x*y^T + A.
    #[allow(clippy::too_many_arguments)]
    pub fn geru<T: GpuVecComplex>(l: Layout, m: usize, n: usize, alpha: T, x: &[T], incx: usize, y: &[T],
                                  incy: usize, a: &mut [T], lda: usize) {
        let mut e = RbError::default();
        must(unsafe { T::ger_raw(false, layout(l), m, n, alpha, x, incx, y, incy, a, lda, &mut e) }, &e)
    }

    /// Drop-in for `rblas::complex2::gerc` (`src/complex2.rs:97-110`): A := alpha*x*y^H + A.
    #[allow(clippy::too_many_arguments)]
    pub fn gerc<T: GpuVecComplex>(l: Layout, m: usize, n: usize, alpha: T, x: &[T], incx: usize, y: &[T],
                                  incy: usize, a: &mut [T], lda: usize) {
        let mut e = RbError::default();
        must(unsafe { T::ger_raw(true, layout(l), m, n, alpha, x, incx, y, incy, a, lda, &mut e) }, &e)
    }
}

#[cfg(test)]
mod tests {
    use super::*;

    /// The error contract of rblas's own try_gemm test (`src/level3.rs:
    /// 590-639`: a short leading dimension, then a short C slice): the same
    /// `BlasError` for the same arguments, found before any device work.
    #[test]
    fn try_gemm_reports_rblas_errors() {
        let a = vec![0.0f64; 6];
        let b = vec![0.0f64; 6];
        let mut c = vec![0.0f64; 4];
        let r = level3::try_gemm(Layout::ColMajor, Transpose::None, Transpose::None, 2, 2, 3, 1.0, &a, 1, &b, 3, 0.0,
                                 &mut c, 2);
        assert_eq!(r, Err(BlasError::InvalidLeadingDim { which: "a", got: 1, min: 2 }));
        let r = level3::try_gemm(Layout::ColMajor, Transpose::None, Transpose::None, 2, 2, 3, 1.0, &a[..5], 2, &b, 3,
                                 0.0, &mut c, 2);
        assert_eq!(r, Err(BlasError::BufferTooSmall { which: "a", got: 5, need: 6 }));
    }

    #[test]
    fn symm_known_answer() {
        // A = [[1, 2], [2, 3]] from its upper triangle, B = [[1, 1], [1, 2]]:
        // A*B = [[3, 5], [5, 8]] exactly (column-major below)
        let a = [1.0f64, 0.0, 2.0, 3.0];
        let b = [1.0f64, 1.0, 1.0, 2.0];
        let mut c = [0.0f64; 4];
        level3::symm(Side::Left, Uplo::Upper, 2, 2, 1.0, &a, 2, &b, 2, 0.0, &mut c, 2);
        assert_eq!(c, [3.0, 5.0, 5.0, 8.0]);
    }
}
