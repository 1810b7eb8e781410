// Reference-wave calibration applied to the reconstructed fields
// (digHolo.cpp:6729-6830, 8233-8285, 8736-8758, 8770-8782).
//
// The stored factors of each calibration item (a frame-sized complex array,
// digHoloConfigSetRefCalibration*) pass through the batch path as a complex
// frame with the frames' FFT windows: a c2c FFT of each polarisation's window,
// the Fourier window placed around kx = ky = 0 (the window bounds at zero tilt
// for a c2c plane, so not held to the positive-kx half), the aperture mask
// centred there, no beam-centre phase, the inverse pixel sinc, the batch
// calibration of the item's index, the normalisation
// sqrt(res / (W H)) / sqrt(W H ifftLength), and an IFFT of the field's size
// (low resolution: the window fftshifted into an h x w plane; full
// resolution: at its own frequencies in the H x W plane).  The resulting
// plane [pol][ny][nx] multiplies the IFFT output of every frame before the
// field statistics and the tilt removal, inside the inverse kernels that
// carry it (k_inverse, k_inverse_dft, and k_field_big for full-resolution
// fields beyond one block; the 512-wide band kernel leaves them to it).
//
// Item of a frame: 0 for a batch of one wavelength; in a multi-wavelength
// batch, the sub-batch's wavelength index modulo the item count (the
// reference takes it from the first frame of each of its thread chunks,
// digHolo.cpp:8746-8750).  Item c is computed at the wavelength its index
// maps to (WavelengthOrderingCalc, digHolo.cpp:2656-2700), with window bounds
// over the batch's wavelength range when there is more than one item.
#include <cmath>
#include <cstring>

#include "dh_object.h"

cudaError_t dh_launch_cal_dft(const DhCalDft& q, cudaStream_t s);
size_t dh_inverse_smem_bytes(const DhInvParams& p);
size_t dh_inverse_dft_smem_bytes(int w, int h, int G);

namespace dh {

static const float PI_F_CAL = 3.14159265358979323846264338327950288f;   // digHolo.cpp:89
static const float UNIT_ANGLE_CAL = PI_F_CAL / 180.0f;                  // DIGHOLO_UNIT_ANGLE, digHolo.h:192

namespace {

// Window corners of the calibration's Fourier window: digHoloIFFT_GetWindowBounds
// without zernCoefs (tilt 0) and r2c = 0 (digHolo.cpp:7868-8048, 6812-6818).
void calWindowCorners(const Config& c, int P, const Geometry& g, float lamStart, float lamStop, int* SX, int* SY) {
    const float k0Max = 2 * PI_F_CAL / (fmaxf(lamStart, lamStop));
    const float k0Min = 2 * PI_F_CAL / (fminf(lamStart, lamStop));
    const float dkx = g.kx[1] - g.kx[0];
    const float dky = g.ky[1] - g.ky[0];
    const float r0 = c.apertureSize * UNIT_ANGLE_CAL;
    const float maxEX = (float)((r0 * k0Max) / dkx + g.W / 2.0);
    const float maxEY = (float)((r0 * k0Max) / dky + g.H / 2.0);
    const float minSX = (float)(((-r0) * k0Min) / dkx + g.W / 2.0);
    const float minSY = (float)(((-r0) * k0Min) / dky + g.H / 2.0);
    const int cxw = (int)std::round((maxEX + minSX) / 4.0) * 2;
    const int cyw = (int)std::round((maxEY + minSY) / 4.0) * 2;
    int w = (int)(16 * std::ceil((1.0f * (int)(maxEX - minSX + 1)) / 16));
    int h = (int)(16 * std::ceil((1.0f * (int)(maxEY - minSY + 1)) / 16));
    if (w < 16) w = 16;
    if (h < 16) h = 16;
    for (int p = 0; p < P; p++) {
        int sx = (int)(cxw - w / 2.0);
        if (sx < 0) sx = 0;
        if (sx + w > g.W) sx = g.W - w;
        SX[p] = sx;
        SY[p] = (int)(cyw - h / 2.0);
    }
}

float xcscF(float x) { return x == 0.f ? 1.0f : (float)((double)x / sin((double)x)); }

template <typename T>
void put(std::vector<unsigned char>& k, T v) {
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&v);
    k.insert(k.end(), b, b + sizeof(T));
}

int posMod(int a, int n) {
    const int r = a % n;
    return r < 0 ? r + n : r;
}

}  // namespace

bool objRefCalApplies(const Object& o) {
    return o.refCalEnabled && o.refCalCount > 0 && !o.refCal.empty() && o.refCalWidth == o.cfg.frameWidth &&
           o.refCalHeight == o.cfg.frameHeight;
}

// The kernels that carry the calibration: k_inverse (power-of-two fields
// whose shared memory fits), k_inverse_dft (low-resolution fields, planes in
// shared memory or global scratch) and k_field_big (full-resolution fields
// beyond one block): every shape this build processes.
int objRefCalCheckShape(Object& o, const DhInvParams& ip) {
    (void)o;
    (void)ip;
    return ERR_SUCCESS;
}

// Planes [pol][ny][nx] of calibration item `item` for the geometry in use.
int objRefCalPlanes(Object& o, int item, const float2** out, bool lookupOnly) {
    *out = nullptr;
    const Config& c = o.useSnaps ? o.ifftSnap : o.cfg;
    const Geometry& g = o.geo;
    const int P = o.polCount, W = g.W, H = g.H, w = g.w, h = g.h, nx = g.nx, ny = g.ny;
    const int count = o.refCalCount;
    const bool lowres = c.resolutionIdx != 0;
    item %= count;
    // wavelength of this item and the window's wavelength range
    const int Lw = o.sweepLambda >= 0 ? (int)o.wavelengths.size() : 1;
    const float centre = o.sweepLambda >= 0 ? o.sweepCentre : c.wavelengthCentre;
    float lam = centre;
    if (Lw > 1) {
        int li;
        if (c.wavelengthOrdering[0] == 0) {
            li = item % Lw;
        } else {
            const int sub = count / Lw;
            li = sub ? item / sub : 0;
        }
        lam = o.wavelengths[std::min(li, Lw - 1)];
    }
    const float lamStart = (count == 1 || Lw == 1) ? centre : o.wavelengths[0];
    const float lamStop = (count == 1 || Lw == 1) ? centre : o.wavelengths[Lw - 1];
    int SXc[POLMAX] = {0, 0}, SYc[POLMAX] = {0, 0};
    calWindowCorners(c, P, g, lamStart, lamStop, SXc, SYc);
    // batch calibration of the item's index, as the caller set it
    const std::vector<float>& bc = o.batchCalCaller ? *o.batchCalCaller : o.batchCal;
    const int bcCount = o.batchCalCaller ? o.batchCalCallerCount : o.batchCalCount;
    const int bcPol = o.batchCalCaller ? o.batchCalCallerPol : o.batchCalPolCount;
    std::vector<float2> ufac(P, make_float2(1.f, 0.f));
    if (o.batchCalEnabled && bcCount > 0 && bcPol > 0 && !bc.empty()) {
        for (int p = 0; p < P; p++) {
            const size_t k = ((size_t)(p % bcPol) * bcCount + (item % bcCount)) * 2;
            ufac[p] = make_float2(bc[k], bc[k + 1]);
        }
    }
    std::vector<unsigned char> key;
    put(key, o.refCalGen); put(key, item); put(key, P); put(key, W); put(key, H); put(key, w); put(key, h);
    put(key, nx); put(key, ny); put(key, (int)lowres); put(key, lam); put(key, c.apertureSize);
    put(key, c.pixelSize); put(key, c.fillFactorCorrection); put(key, c.frameWidth); put(key, c.frameHeight);
    for (int p = 0; p < P; p++) {
        put(key, g.cx[p]); put(key, g.cy[p]); put(key, SXc[p]); put(key, SYc[p]); put(key, ufac[p].x); put(key, ufac[p].y);
    }
    for (auto& e : o.refCalPlanes)
        if (e->key == key) {
            *out = e->planes.as<float2>();
            return ERR_SUCCESS;
        }
    if (lookupOnly)
        return fail(o, ERR_ERROR, "no-alloc path: process one batch with this calibration first (that call computes its planes)");
    if (o.refCalPlanes.size() >= 8) o.refCalPlanes.erase(o.refCalPlanes.begin());
    int r = objInitDevice(o);
    if (r) return r;
    // the stored factors on the device, once per setter call
    const size_t frame = (size_t)o.refCalWidth * o.refCalHeight;
    if (o.refCalFramesGen != o.refCalGen) {
        DH_CUDA(o, o.dRefCalFrames.ensure(o.refCal.size() * sizeof(float)));
        DH_CUDA(o, cudaMemcpyAsync(o.dRefCalFrames.ptr, o.refCal.data(), o.refCal.size() * sizeof(float),
                                   cudaMemcpyHostToDevice, o.stream));
        o.refCalFramesGen = o.refCalGen;
    }
    // index tables and window factors (float32 as digHoloCopyWindow forms them)
    const float k0 = 2 * PI_F_CAL / lam;
    const float kr = k0 * sinf(c.apertureSize * UNIT_ANGLE_CAL);
    const float r02 = kr * kr;
    const float norm0 = sqrtf((float)((1.0 * nx * ny) / (1.0 * W * H)));
    const double ifftLength = lowres ? 1.0 * w * h : 1.0 * W * H;
    const float norm = (float)(norm0 / sqrt((1.0 * W * H) * ifftLength));
    const float halfPixel = 0.5f * c.pixelSize;
    const float kyShift = fabsf((g.ky[1] - g.ky[0]) * H);
    std::vector<int> colIdx((size_t)P * w), rowIdx((size_t)P * h), destCol((size_t)P * w), destRow((size_t)P * h);
    std::vector<float> fac((size_t)P * h * w, 0.f);
    for (int p = 0; p < P; p++) {
        for (int i = 0; i < w; i++) {
            int col = i + SXc[p] - W / 2;
            if (col < 0) col += W;
            const bool ok = col >= 0 && col < W;
            colIdx[(size_t)p * w + i] = ok ? col : 0;
            destCol[(size_t)p * w + i] = lowres ? (i + w / 2) % w : (ok ? col : 0);
        }
        for (int j = 0; j < h; j++) {
            const int jSY = j + SYc[p];
            const int row = posMod(jSY + H / 2, H);
            rowIdx[(size_t)p * h + j] = row;
            destRow[(size_t)p * h + j] = lowres ? (j + h / 2) % h : row;
            const float ky = g.ky[row];
            const float shift = jSY < 0 ? kyShift : (jSY > H ? -kyShift : 0.0f);
            volatile float dky = ky - (0.0f + shift);
            volatile float dky2 = dky * dky;
            for (int i = 0; i < w; i++) {
                int col = i + SXc[p] - W / 2;
                if (col < 0) col += W;
                if (col < 0 || col >= W) continue;
                const float kx = g.kx[col];
                volatile float dkx2 = kx * kx;
                const float dr2 = dkx2 + dky2;
                const float env = c.fillFactorCorrection ? xcscF(kx * halfPixel) * xcscF(ky * halfPixel) : 1.0f;
                fac[((size_t)p * h + j) * w + i] = (dr2 <= r02) ? env * norm : 0.0f;
            }
        }
    }
    // device tables: colIdx, rowIdx, destCol, destRow (int), ufac (float2), fac (float)
    const size_t nInt = colIdx.size() + rowIdx.size() + destCol.size() + destRow.size();
    const size_t tabBytes = nInt * sizeof(int) + ufac.size() * sizeof(float2) + fac.size() * sizeof(float) + 64;
    DH_CUDA(o, o.dRefCalTables.ensure(tabBytes));
    std::vector<unsigned char> tab(tabBytes, 0);
    size_t off = 0;
    auto stage = [&](const void* src, size_t bytes) {
        const size_t at = off;
        memcpy(tab.data() + off, src, bytes);
        off = (off + bytes + 15) & ~(size_t)15;
        return at;
    };
    const size_t oCol = stage(colIdx.data(), colIdx.size() * sizeof(int));
    const size_t oRow = stage(rowIdx.data(), rowIdx.size() * sizeof(int));
    const size_t oDCol = stage(destCol.data(), destCol.size() * sizeof(int));
    const size_t oDRow = stage(destRow.data(), destRow.size() * sizeof(int));
    const size_t oUfac = stage(ufac.data(), ufac.size() * sizeof(float2));
    const size_t oFac = stage(fac.data(), fac.size() * sizeof(float));
    DH_CUDA(o, cudaMemcpyAsync(o.dRefCalTables.ptr, tab.data(), off, cudaMemcpyHostToDevice, o.stream));
    const char* T = o.dRefCalTables.as<char>();
    // scratch: R [P][H][w], V [P][h][w], S [P][h][nx]
    const size_t nR = (size_t)P * H * w, nV = (size_t)P * h * w, nS = (size_t)P * h * nx;
    DH_CUDA(o, o.dRefCalScratch.ensure((nR + nV + nS) * sizeof(float2)));
    float2* R = o.dRefCalScratch.as<float2>();
    float2* V = R + nR;
    float2* S = V + nV;
    auto entry = std::make_unique<Object::RefCalPlanes>();
    DH_CUDA(o, entry->planes.ensure((size_t)P * ny * nx * sizeof(float2)));
    float2* planes = entry->planes.as<float2>();
    const float2* frames = o.dRefCalFrames.as<float2>() + (size_t)item * frame;
    // 1. rows of each polarisation's FFT window: R[y][i] = sum_x cal[y][x] e^{-2 pi i col(i) x / W}
    for (int p = 0; p < P; p++) {
        DhCalDft q;
        memset(&q, 0, sizeof(q));
        q.in = frames + (size_t)g.cy[p] * o.refCalWidth + g.cx[p];
        q.inU = 0; q.inA = o.refCalWidth; q.inB = 0; q.inK = 1;
        q.out = R + (size_t)p * H * w;
        q.U = 1; q.A = H; q.B = w; q.K = W;
        q.freqOut = reinterpret_cast<const int*>(T + oCol) + (size_t)p * w;
        q.outOnA = 0;
        q.fP = 1; q.N = W; q.sign = -1;
        DH_CUDA(o, dh_launch_cal_dft(q, o.stream));
    }
    // 2. columns at the window's rows, then the batch factor and the window factors
    {
        DhCalDft q;
        memset(&q, 0, sizeof(q));
        q.in = R; q.inU = (long long)H * w; q.inA = 0; q.inB = 1; q.inK = w;
        q.out = V;
        q.U = P; q.A = h; q.B = w; q.K = H;
        q.freqOut = reinterpret_cast<const int*>(T + oRow);
        q.outOnA = 1;
        q.fP = P; q.N = H; q.sign = -1;
        q.ufac = reinterpret_cast<const float2*>(T + oUfac);
        q.fac = reinterpret_cast<const float*>(T + oFac);
        DH_CUDA(o, dh_launch_cal_dft(q, o.stream));
    }
    // 3. inverse along the window's columns to the field's x: S[j][x]
    {
        DhCalDft q;
        memset(&q, 0, sizeof(q));
        q.in = V; q.inU = (long long)h * w; q.inA = w; q.inB = 0; q.inK = 1;
        q.out = S;
        q.U = P; q.A = h; q.B = nx; q.K = w;
        q.freqK = reinterpret_cast<const int*>(T + oDCol);
        q.fP = P; q.N = nx; q.sign = 1;
        DH_CUDA(o, dh_launch_cal_dft(q, o.stream));
    }
    // 4. inverse along the window's rows to the field's y: planes[y][x]
    {
        DhCalDft q;
        memset(&q, 0, sizeof(q));
        q.in = S; q.inU = (long long)h * nx; q.inA = 0; q.inB = 1; q.inK = nx;
        q.out = planes;
        q.U = P; q.A = ny; q.B = nx; q.K = h;
        q.freqK = reinterpret_cast<const int*>(T + oDRow);
        q.outOnA = 1;
        q.fP = P; q.N = ny; q.sign = 1;
        DH_CUDA(o, dh_launch_cal_dft(q, o.stream));
    }
    // the tables and the scratch are reused by the next item: let this one finish
    DH_CUDA(o, cudaStreamSynchronize(o.stream));
    entry->key = std::move(key);
    *out = planes;
    o.refCalPlanes.push_back(std::move(entry));
    return ERR_SUCCESS;
}

// digHoloConfigGetRefCalibrationFields: every item's planes for the geometry
// of the last batch, [item][pol][ny][nx], with the field's axes.
int objRefCalFieldsToHost(Object& o) {
    if (!objRefCalApplies(o) || !o.preparedValid || o.geo.nx <= 0)
        return fail(o, ERR_NULLPOINTER, "no reference-wave calibration applied to a processed batch");
    const size_t per = (size_t)o.polCount * o.geo.nx * o.geo.ny;
    if (!o.hRefCalFields.ensure((size_t)o.refCalCount * per * sizeof(float2)))
        return fail(o, ERR_MEMORYALLOCATION, "host calibration buffer");
    for (int item = 0; item < o.refCalCount; item++) {
        const float2* planes = nullptr;
        int r = objRefCalPlanes(o, item, &planes, false);
        if (r) return r;
        DH_CUDA(o, cudaMemcpyAsync(o.hRefCalFields.as<float2>() + (size_t)item * per, planes, per * sizeof(float2),
                                   cudaMemcpyDeviceToHost, o.stream));
    }
    DH_CUDA(o, cudaStreamSynchronize(o.stream));
    o.hRefCalX = o.geo.x;
    o.hRefCalY = o.geo.y;
    return ERR_SUCCESS;
}

}  // namespace dh
