"""Complex128 field transport (oracle).

Restates the reference's complex mirrors ``tests/ad/_reference_fields.py:17-337``
(free space, slab Fresnel, reflection sequence, Rouard stack, transmission
sequence) which in turn mirror ``native/channel/kernels/fields.cu:36-204`` and
RayD's ``field_transport``.  All arrays are NumPy float64 / complex128 and
vectorised over the leading row axis.

Test infrastructure only: the tests, the smoke check and the benchmark's CPU
baseline call it as the checker; the product path never does.
"""

from __future__ import annotations

import numpy as np

SPEED_OF_LIGHT = 299792458.0
VACUUM_PERMITTIVITY = 8.8541878128e-12
VACUUM_PERMEABILITY = 1.25663706212e-6
EPS = 1.0e-10  # utd::UTD_EPS (_reference_fields.py:12)
SMALL_EPS = 1.0e-6  # utd::UTD_SMALL_EPS (_reference_fields.py:13)
POL_TE = 0
POL_TM = 1


def norm(v: np.ndarray) -> np.ndarray:
    return np.sqrt(np.sum(v * v, axis=-1))


def dot(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.sum(a * b, axis=-1)


def safe_normalize(v: np.ndarray, fallback: np.ndarray) -> np.ndarray:
    """``_reference_fields.py:17-22``."""
    n = norm(v)[..., None]
    fb = fallback / (norm(fallback)[..., None] + EPS)
    return np.where(n > SMALL_EPS, v / (n + EPS), fb)


def stable_perp_basis(ray_dir: np.ndarray, preferred: np.ndarray) -> np.ndarray:
    """``_reference_fields.py:25-31``."""
    proj = preferred - ray_dir * dot(preferred, ray_dir)[..., None]
    e_z = np.array([0.0, 0.0, 1.0])
    e_y = np.array([0.0, 1.0, 0.0])
    alt = np.where((np.abs(ray_dir[..., 2:3]) < 0.9), e_z, e_y)
    alt_proj = alt - ray_dir * dot(alt, ray_dir)[..., None]
    return safe_normalize(proj, alt_proj)


def transverse_project(ray_dir: np.ndarray, preferred: np.ndarray) -> np.ndarray:
    """Unnormalised transverse projection ``p - (p.k)k`` (``_reference_fields.py:34-37``)."""
    return preferred - ray_dir * dot(preferred, ray_dir)[..., None]


def project(value: np.ndarray, axis: np.ndarray) -> np.ndarray:
    return np.sum(value * axis, axis=-1)


def outputs(value: np.ndarray, rx_axis: np.ndarray, tx_power: np.ndarray) -> dict:
    """``_reference_fields.py:48-61``."""
    coefficient = project(value, rx_axis)
    path_field = coefficient * np.sqrt(np.maximum(tx_power, 0.0))
    return {
        "field_vector": value,
        "coefficient": coefficient,
        "path_field": path_field,
        "path_gain": path_field.real ** 2 + path_field.imag ** 2,
    }


def wave_number(frequency: float) -> float:
    return 2.0 * np.pi * frequency / SPEED_OF_LIGHT


def free_space(source, target, tx_power, tx_pol, rx_pol, frequency) -> dict:
    """``_reference_fields.py:64-82``; ``fields.cu:36-82``."""
    offset = target - source
    distance = norm(offset)
    e_z = np.broadcast_to(np.array([0.0, 0.0, 1.0]), offset.shape)
    direction = safe_normalize(offset, e_z)
    tx_axis = transverse_project(direction, tx_pol)
    rx_axis = transverse_project(direction, rx_pol)
    k = wave_number(frequency)
    amplitude = 1.0 / (2.0 * max(k, SMALL_EPS) * np.maximum(distance, EPS))
    carrier = amplitude * np.exp(-1.0j * k * distance)
    value = tx_axis * carrier[..., None]
    out = outputs(value, rx_axis, tx_power)
    out["path_length_m"] = distance
    out["delay_s"] = distance / SPEED_OF_LIGHT
    out["direction"] = direction
    return out


def slab_fresnel(cos_theta, eps_r, sigma_e, mu_r, gain, thickness, frequency):
    """Thin-slab Fabry-Perot reflection (``_reference_fields.py:85-115``)."""
    omega = max(2.0 * np.pi * frequency, SMALL_EPS)
    wavelength = SPEED_OF_LIGHT / frequency
    ct = np.clip(np.abs(cos_theta), SMALL_EPS, 1.0)
    sin2 = np.maximum(1.0 - ct * ct, 0.0)
    eta = np.maximum(eps_r, SMALL_EPS) - 1.0j * np.maximum(sigma_e, 0.0) / (omega * VACUUM_PERMITTIVITY)
    mu = np.maximum(mu_r, SMALL_EPS)
    root = np.sqrt(eta * mu - sin2 + 0.0j)
    mu_ct = mu * ct
    eta_ct = eta * ct
    interface_te = (mu_ct - root) / (mu_ct + root)
    interface_tm = (eta_ct - root) / (eta_ct + root)
    q = root * (2.0 * np.pi * np.maximum(thickness, 0.0) / max(wavelength, SMALL_EPS))
    phase = np.exp(-2.0j * q)
    r_te = gain * (interface_te * (1.0 - phase)) / (1.0 - interface_te * interface_te * phase)
    r_tm = gain * (interface_tm * (1.0 - phase)) / (1.0 - interface_tm * interface_tm * phase)
    return r_te, r_tm


def halfspace_fresnel(cos_theta, eps_r, sigma_e, mu_r, gain, frequency):
    """Interface (half-space) Fresnel coefficients ``gain * (r_te, r_tm)``: the
    slab law above without the Fabry-Perot layer term.  The wedge faces of
    first-order diffraction take this form, with the cosine given by the wedge
    angles (the reference's design notes,
    ``docs/dev/plans/07-channel-native-differentiable-solver-plan.md:57``)."""
    omega = max(2.0 * np.pi * frequency, SMALL_EPS)
    ct = np.clip(np.abs(cos_theta), SMALL_EPS, 1.0)
    sin2 = np.maximum(1.0 - ct * ct, 0.0)
    eta = np.maximum(eps_r, SMALL_EPS) - 1.0j * np.maximum(sigma_e, 0.0) / (omega * VACUUM_PERMITTIVITY)
    mu = np.maximum(mu_r, SMALL_EPS)
    root = np.sqrt(eta * mu - sin2 + 0.0j)
    r_te = gain * (mu * ct - root) / (mu * ct + root)
    r_tm = gain * (eta * ct - root) / (eta * ct + root)
    return r_te, r_tm


def reflection_sequence(source, target, positions, normals, tx_power, tx_pol, rx_pol,
                        eps_r, sigma_e, mu_r, gain, thickness, frequency) -> dict:
    """General-depth specular chain (``_reference_fields.py:118-186``; ``fields.cu:113-204``).

    ``positions``/``normals`` are ``(N, D, 3)``; material arrays ``(N, D)``.
    Path length is summed in float64 over the segments.
    """
    depth = positions.shape[1]
    e_z = np.broadcast_to(np.array([0.0, 0.0, 1.0]), source.shape)
    previous = source
    incident = safe_normalize(positions[:, 0] - previous, e_z)
    tx_axis = transverse_project(incident, tx_pol)
    value = tx_axis.astype(np.complex128)
    total_length = np.zeros(source.shape[0])
    outgoing = incident
    for bounce in range(depth):
        hit = positions[:, bounce]
        segment = hit - previous
        incident = safe_normalize(segment, outgoing)
        total_length = total_length + norm(segment)
        normal = safe_normalize(normals[:, bounce], e_z)
        flip = dot(incident, normal) > 0.0
        oriented = np.where(flip[:, None], -normal, normal)
        dot_in = dot(incident, oriented)
        reflected = safe_normalize(incident - oriented * (2.0 * dot_in)[:, None], -incident)
        s_axis = safe_normalize(np.cross(oriented, incident), stable_perp_basis(incident, oriented))
        p_in = safe_normalize(np.cross(s_axis, incident), stable_perp_basis(incident, s_axis))
        p_out = safe_normalize(np.cross(s_axis, reflected), stable_perp_basis(reflected, s_axis))
        r_te, r_tm = slab_fresnel(np.abs(dot_in), eps_r[:, bounce], sigma_e[:, bounce], mu_r[:, bounce],
                                  gain[:, bounce], thickness[:, bounce], frequency)
        e_s = project(value, s_axis)
        e_p = project(value, p_in)
        value = s_axis * (r_te * e_s)[:, None] + p_out * (r_tm * e_p)[:, None]
        outgoing = reflected
        previous = hit
    final_offset = target - previous
    final_direction = safe_normalize(final_offset, outgoing)
    total_length = total_length + norm(final_offset)
    k = wave_number(frequency)
    amplitude = 1.0 / (2.0 * k * np.maximum(total_length, EPS))
    value = value * (amplitude * np.exp(-1.0j * k * total_length))[:, None]
    rx_axis = transverse_project(final_direction, rx_pol)
    out = outputs(value, rx_axis, tx_power)
    out["path_length_m"] = total_length
    out["delay_s"] = total_length / SPEED_OF_LIGHT
    out["direction"] = final_direction
    return out


def stack_rt(cos_theta: float, thickness, eps_r, sigma_e, mu_r, frequency: float, pol: int):
    """Backward Rouard recursion for one wall (``_reference_fields.py:196-273``).

    Layer arrays are ordered entry -> exit; returns ``(r, t)``.
    """
    omega = max(2.0 * np.pi * frequency, SMALL_EPS)
    ct = min(max(abs(cos_theta), SMALL_EPS), 1.0)
    sin2 = max(1.0 - ct * ct, 0.0)
    k_entry = omega / SPEED_OF_LIGHT
    k_par = k_entry * np.sqrt(sin2)

    def admittance(eps_abs, mu_abs, k_z):
        if pol == POL_TE:
            return k_z / (mu_abs * omega)
        return (eps_abs * omega) / k_z

    kz_entry = complex(k_entry * ct)
    y_entry = admittance(complex(VACUUM_PERMITTIVITY), complex(VACUUM_PERMEABILITY), kz_entry)
    y_exit = y_entry
    count = len(thickness)
    if count == 0:
        return 0.0j, 1.0 + 0.0j

    def medium(i):
        eps_abs = complex(VACUUM_PERMITTIVITY * max(eps_r[i], SMALL_EPS), -max(sigma_e[i], 0.0) / omega)
        mu_abs = complex(VACUUM_PERMEABILITY * max(mu_r[i], SMALL_EPS))
        k = np.sqrt(eps_abs * mu_abs) * omega
        k_z = np.sqrt(k * k - complex(k_par * k_par))
        return eps_abs, mu_abs, k_z

    eps_b, mu_b, kz_below = medium(count - 1)
    y_below = admittance(eps_b, mu_b, kz_below)
    r_total = (y_below - y_exit) / (y_below + y_exit)
    t_total = 2.0 * y_below / (y_below + y_exit)
    for layer in range(count - 1, -1, -1):
        phase = np.exp(-1.0j * kz_below * max(thickness[layer], 0.0))
        phase2 = phase * phase
        if layer > 0:
            eps_a, mu_a, kz_above = medium(layer - 1)
            y_above = admittance(eps_a, mu_a, kz_above)
        else:
            kz_above = kz_entry
            y_above = y_entry
        r_top = (y_above - y_below) / (y_above + y_below)
        t_top = 2.0 * y_above / (y_above + y_below)
        loop = phase2 * r_total
        denominator = 1.0 + r_top * loop
        r_total = (r_top + loop) / denominator
        t_total = t_top * phase * t_total / denominator
        kz_below = kz_above
        y_below = y_above
    return r_total, t_total


def transmission_sequence(source, target, normals, material_ids, depth, tx_power, tx_pol, rx_pol,
                          layers: list, frequency: float) -> dict:
    """Straight thin-sheet chain (``_reference_fields.py:276-337``).

    ``normals`` ``(N, D, 3)``; ``material_ids`` ``(N, D)``; ``depth`` ``(N,)``
    valid wall count; ``layers[m]`` is a tuple of arrays
    ``(thickness, eps_r, sigma_e, mu_r)`` for material ``m``.
    """
    count = source.shape[0]
    e_z = np.broadcast_to(np.array([0.0, 0.0, 1.0]), source.shape)
    offset = target - source
    total_length = norm(offset)
    direction = safe_normalize(offset, e_z)
    tx_axis = transverse_project(direction, tx_pol)
    rx_axis = transverse_project(direction, rx_pol)
    k = wave_number(frequency)
    values = np.zeros((count, 3), dtype=np.complex128)
    carrier_out = np.zeros(count)
    for i in range(count):
        value = tx_axis[i].astype(np.complex128)
        carrier = total_length[i]
        d = direction[i]
        for wall in range(int(depth[i])):
            m = int(material_ids[i, wall])
            n = safe_normalize(normals[i, wall][None, :], np.array([[0.0, 0.0, 1.0]]))[0]
            if float(np.dot(d, n)) > 0.0:
                n = -n
            cos_theta = min(max(abs(float(np.dot(d, n))), SMALL_EPS), 1.0)
            th, er, sg, mr = layers[m]
            _, t_te = stack_rt(cos_theta, th, er, sg, mr, frequency, POL_TE)
            _, t_tm = stack_rt(cos_theta, th, er, sg, mr, frequency, POL_TM)
            s_axis = safe_normalize(np.cross(n, d)[None, :], stable_perp_basis(d[None, :], n[None, :]))[0]
            p_axis = safe_normalize(np.cross(s_axis, d)[None, :], stable_perp_basis(d[None, :], s_axis[None, :]))[0]
            e_s = np.sum(value * s_axis)
            e_p = np.sum(value * p_axis)
            value = s_axis * (t_te * e_s) + p_axis * (t_tm * e_p)
            carrier = carrier - float(np.sum(np.maximum(th, 0.0))) * cos_theta
        amplitude = 1.0 / (2.0 * k * max(total_length[i], EPS))
        values[i] = value * (amplitude * np.exp(-1.0j * k * carrier))
        carrier_out[i] = carrier
    out = outputs(values, rx_axis, tx_power)
    out["path_length_m"] = total_length
    out["delay_s"] = total_length / SPEED_OF_LIGHT
    out["direction"] = direction
    return out


def project_complex3(field_vector, direction, rx_pol) -> dict:
    """Receiver projection (``fields.cu:84-105``)."""
    rx_axis = transverse_project(direction, rx_pol)
    coefficient = project(field_vector, rx_axis)
    return {"coefficient": coefficient, "path_gain": np.abs(coefficient) ** 2}
